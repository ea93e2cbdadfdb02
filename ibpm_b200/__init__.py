"""B200-native IBPM time step.

Host side of the C ABI in ``include/ibpm_b200.h``; the names mirror the
reference's classes (paths inside the reference project):

* ``Grid``                 src/Grid.h
* ``State``                src/State.h (omega, q, f, timestep, time; computeNetForce)
* ``NavierStokesModel``    src/NavierStokesModel.h (Reynolds number, base flow, geometry)
* ``NonlinearIBSolver``    src/IBSolver.h (init/load/save/advance)
* ``PoissonSolver`` / ``HelmholtzSolver``  src/EllipticSolver.h

The compute path is the CUDA library ``libibpm_b200.so``; nothing here
computes on the CPU.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import geometry as _geometry
from ._native import (PRECISIONS, PRECONDS, SCHEMES, IbgError, check, ibg_body, ibg_grid, ibg_params, lib)

__all__ = ["Grid", "State", "NavierStokesModel", "NonlinearIBSolver", "IbgError", "geometry"]
geometry = _geometry


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class Grid:
    """Grid(nx, ny, ngrid, length, xoffset, yoffset) (src/Grid.h:36-44)."""
    nx: int
    ny: int
    ngrid: int
    length: float
    xoffset: float
    yoffset: float

    @property
    def dx(self) -> float:
        return self.length / self.nx

    @property
    def n_scalar(self) -> int:
        return self.ngrid * (self.nx - 1) * (self.ny - 1)

    @property
    def n_flux(self) -> int:
        return self.ngrid * (2 * self.nx * self.ny + self.nx + self.ny)

    def scalar(self) -> np.ndarray:
        return np.zeros((self.ngrid, self.nx - 1, self.ny - 1))

    def flux(self) -> np.ndarray:
        return np.zeros((self.ngrid, 2 * self.nx * self.ny + self.nx + self.ny))


@dataclass
class State:
    """State (src/State.h): vorticity, flux, boundary force, timestep, time."""
    grid: Grid
    npoints: int
    omega: np.ndarray = None
    q: np.ndarray = None
    f: np.ndarray = None
    timestep: int = 0
    time: float = 0.0

    def __post_init__(self):
        if self.omega is None:
            self.omega = self.grid.scalar()
        if self.q is None:
            self.q = self.grid.flux()
        if self.f is None:
            self.f = np.zeros(2 * self.npoints)

    def computeNetForce(self):
        """State::computeNetForce (src/State.cc:53-63)."""
        n = self.npoints
        dx2 = self.grid.dx * self.grid.dx
        return float(self.f[:n].sum() * dx2), float(self.f[n:].sum() * dx2)


@dataclass
class NavierStokesModel:
    """NavierStokesModel(grid, geometry, Re, q_potential) (src/NavierStokesModel.h:35-122);
    the base flow is uniform with magnitude `u_mag` and angle `alpha` (radians).
    ``ubf=True`` is the CLI's unsteady base flow (src/ibpm.cc:166-178): the
    single body's motion is carried by the base flow instead."""
    grid: Grid
    geom: _geometry.Geometry
    Re: float
    u_mag: float = 1.0
    alpha: float = 0.0
    ubf: bool = False

    def getAlpha(self) -> float:
        return 1.0 / self.Re

    def getNumPoints(self) -> int:
        return self.geom.num_points


class NonlinearIBSolver:
    """NonlinearIBSolver(grid, model, dt, scheme, tol) (src/IBSolver.h:69-90) on the GPU.

    ``advance(x)`` keeps the reference's contract (the host State is valid
    after every call); ``advance_resident(n)`` steps the device-resident state
    without host traffic.
    """

    def __init__(self, grid: Grid, model: NavierStokesModel, dt: float, scheme: str = "rk3", tol: float = 1e-7,
                 precision: str = "fp64", stream: Optional[int] = None, cg_max_iter: int = 3000,
                 device: int = -1, precond: str = "none", pc_refresh: int = 10, cg_graph: bool = True,
                 pc_fallback_iter: int = 0):
        self.grid, self.model, self.dt = grid, model, dt
        self.scheme = scheme
        L = lib()
        g = ibg_grid(grid.nx, grid.ny, grid.ngrid, grid.length, grid.xoffset, grid.yoffset)
        self._keep = []
        bodies = (ibg_body * len(model.geom.bodies))()
        for k, b in enumerate(model.geom.bodies):
            xy = np.ascontiguousarray(np.array(b.points, dtype=np.float64).reshape(-1))
            self._keep.append(xy)
            bodies[k].npoints = len(b.points)
            bodies[k].xy = xy.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            bodies[k].xcenter, bodies[k].ycenter = b.center
            bodies[k].motion = b.motion
            for j in range(12):
                bodies[k].params[j] = b.params[j] if j < len(b.params) else 0.0
            if b.table is not None and len(b.table):
                tab = np.ascontiguousarray(np.asarray(b.table, dtype=np.float64).reshape(-1, 7))
                self._keep.append(tab)
                bodies[k].table_rows = tab.shape[0]
                bodies[k].table = tab.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        p = ibg_params(model.Re, dt, SCHEMES[scheme], tol, cg_max_iter, model.u_mag, model.alpha,
                       PRECISIONS[precision], device, PRECONDS[precond], pc_refresh, int(cg_graph),
                       pc_fallback_iter)
        h = ctypes.c_void_p()
        check(L.ibg_create(ctypes.byref(g), len(model.geom.bodies), bodies, ctypes.byref(p),
                           ctypes.c_void_p(stream) if stream else None, ctypes.byref(h)), None)
        self._h = h
        self.npoints = model.geom.num_points
        self._synced = None
        if model.ubf:
            check(L.ibg_set_moving_frame(h), h)

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().ibg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -- IBSolver interface -------------------------------------------------
    def init(self):
        check(lib().ibg_init(self._h), self._h)

    def load(self, basename: str) -> bool:
        return check(lib().ibg_load(self._h, basename.encode()), self._h) == 1

    def save(self, basename: str) -> bool:
        return check(lib().ibg_save(self._h, basename.encode()), self._h) == 1

    def getTimestep(self) -> float:
        return self.dt

    def set_state(self, x: State, with_q: bool = True):
        om = np.ascontiguousarray(x.omega, dtype=np.float64)
        q = np.ascontiguousarray(x.q, dtype=np.float64) if with_q else None
        f = np.ascontiguousarray(x.f, dtype=np.float64)
        check(lib().ibg_set_state(self._h, _ptr(om), _ptr(q), _ptr(f), int(x.timestep), float(x.time)), self._h)
        self._synced = x

    def get_state(self, x: State):
        om = np.empty(x.omega.shape)
        q = np.empty(x.q.shape)
        f = np.empty(x.f.shape)
        ts = ctypes.c_int()
        t = ctypes.c_double()
        check(lib().ibg_get_state(self._h, _ptr(om), _ptr(q), _ptr(f), ctypes.byref(ts), ctypes.byref(t)), self._h)
        x.omega, x.q, x.f, x.timestep, x.time = om, q, f, ts.value, t.value

    # -- inner products and energy (src/VectorOperations.cc:222-412) ---------
    def inner_product(self, a, b, fine_only: bool = False) -> float:
        """InnerProduct (or FineGridInnerProduct) of two Scalars or two Fluxes."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        kind = (2 if a.shape == self.grid.flux().shape else 0) + (1 if fine_only else 0)
        out = ctypes.c_double()
        check(lib().ibg_inner_product(self._h, kind, _ptr(a), _ptr(b), ctypes.byref(out)), self._h)
        return out.value

    def energy(self) -> float:
        """0.5 InnerProduct(q, q) of the device state (OutputEnergy, src/OutputEnergy.cc:29-33)."""
        out = ctypes.c_double()
        check(lib().ibg_energy(self._h, ctypes.byref(out)), self._h)
        return out.value

    # -- the other N(x) forms (src/IBSolver.cc:211-283) ----------------------
    def set_linearized(self, omega0, q0=None):
        """LinearizedIBSolver (one base state) or LinearizedPeriodicIBSolver (a list of
        them, phase = timestep % period).  None restores the nonlinear solver."""
        if omega0 is None:
            check(lib().ibg_set_linearized(self._h, 0, None, None), self._h)
            return
        w = np.ascontiguousarray(np.stack([np.asarray(a, dtype=np.float64) for a in
                                           (omega0 if isinstance(omega0, (list, tuple)) else [omega0])]))
        q = np.ascontiguousarray(np.stack([np.asarray(a, dtype=np.float64) for a in
                                           (q0 if isinstance(q0, (list, tuple)) else [q0])]))
        if w.shape[0] != q.shape[0]:
            raise ValueError("as many base vorticity fields as base flux fields")
        check(lib().ibg_set_linearized(self._h, int(w.shape[0]), _ptr(w), _ptr(q)), self._h)

    def set_adjoint(self, omega0, q0):
        """AdjointIBSolver about the base state (omega0, q0)."""
        w = np.ascontiguousarray(omega0, dtype=np.float64)
        q = np.ascontiguousarray(q0, dtype=np.float64)
        check(lib().ibg_set_adjoint(self._h, _ptr(w), _ptr(q)), self._h)

    def set_sfd(self, chi: float, Delta: float, omega_hat=None):
        """SFDSolver: selective frequency damping with gain chi and filter width Delta."""
        wh = None if omega_hat is None else np.ascontiguousarray(omega_hat, dtype=np.float64)
        check(lib().ibg_set_sfd(self._h, float(chi), float(Delta), _ptr(wh)), self._h)

    def sfd_filtered(self) -> np.ndarray:
        out = np.zeros(self.grid.scalar().shape)
        check(lib().ibg_get_sfd_state(self._h, _ptr(out)), self._h)
        return out

    # -- restart files (State::save / State::load, src/State.cc:65-223) -------
    def save_restart(self, filename: str) -> bool:
        return check(lib().ibg_save_restart(self._h, filename.encode()), self._h) == 1

    def load_restart(self, filename: str) -> bool:
        return check(lib().ibg_load_restart(self._h, filename.encode()), self._h) == 1

    def snapshot(self):
        """Copy the current state for a later restart file without stalling the GPU."""
        check(lib().ibg_snapshot(self._h), self._h)

    def snapshot_save(self, filename: str) -> bool:
        return check(lib().ibg_snapshot_save(self._h, filename.encode()), self._h) == 1

    def update_operators(self, time: float):
        check(lib().ibg_update_operators(self._h, float(time)), self._h)

    def flux_to_velocity(self):
        """FluxToVelocity of the device state's flux: node velocities (u, v), each (ngrid, nx-1, ny-1);
        0 on the coarse interior nodes the reference leaves undefined."""
        g = self.grid
        u = np.empty((g.ngrid, g.nx - 1, g.ny - 1))
        v = np.empty_like(u)
        check(lib().ibg_flux_to_velocity(self._h, _ptr(u), _ptr(v)), self._h)
        return u, v

    def boundary(self):
        """Geometry::getPoints / getVelocities at the last time the bodies were
        moved, as (npoints, 2) arrays of positions and velocities."""
        n = self.model.geom.num_points
        pts = np.empty(2 * n)
        vel = np.empty(2 * n)
        check(lib().ibg_get_boundary(self._h, _ptr(pts), _ptr(vel)), self._h)
        return pts.reshape(2, n).T.copy(), vel.reshape(2, n).T.copy()

    def refresh_state(self, x: State):
        """model->refreshState(x): q from omega on the device."""
        self.set_state(x, with_q=False)
        self.get_state(x)

    def advance(self, x: State):
        """IBSolver::advance(State&) (src/IBSolver.cc:142-149)."""
        if self._synced is not x:
            self.set_state(x)
        check(lib().ibg_advance(self._h, 1), self._h)
        self.get_state(x)

    def advance_resident(self, nsteps: int = 1):
        check(lib().ibg_advance(self._h, int(nsteps)), self._h)

    def force_history(self, n: int) -> np.ndarray:
        out = np.zeros((n, 2))
        k = check(lib().ibg_get_force_history(self._h, n, _ptr(out)), self._h)
        return out[:k]

    def net_force(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        check(lib().ibg_get_net_force(self._h, ctypes.byref(a), ctypes.byref(b)), self._h)
        return a.value, b.value

    def cg_totals(self):
        it, n = ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().ibg_cg_totals(self._h, ctypes.byref(it), ctypes.byref(n)), self._h)
        return it.value, n.value

    def cg_stats(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().ibg_cg_stats(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), self._h)
        return a.value, b.value, c.value

    def stream(self) -> int:
        return lib().ibg_stream(self._h) or 0

    def last_launch_count(self) -> int:
        return int(lib().ibg_last_launch_count(self._h))

    # -- learned preconditioner (no reference counterpart) -----------------
    def lpc_generate(self, nconfig: int, t0: float, t1: float):
        """Training data from this solver's exact force operator: geometry
        features [nconfig, npts, 4] and M / beta [nconfig, m, m] (float32) at
        nconfig body configurations evenly spread over [t0, t1]."""
        P = self.npoints
        m = 2 * P
        geom = np.zeros((nconfig, P, 4), np.float32)
        mb = np.zeros((nconfig, m, m), np.float32)
        check(lib().ibg_lpc_generate(self._h, int(nconfig), float(t0), float(t1), _ptr(geom), _ptr(mb)), self._h)
        return geom, mb

    def lpc_train(self, geom, mb, epochs: int = 200, batch: int = 4, lr: float = 1e-3, seed: int = 0):
        """Fit the network on the device (Adam, FP32) and enable it; returns the
        mean loss of every epoch."""
        geom, mb = (np.ascontiguousarray(a, dtype=np.float32) for a in (geom, mb))
        hist = np.zeros(epochs, np.float32)
        check(lib().ibg_lpc_train(self._h, int(mb.shape[0]), _ptr(geom), _ptr(mb), int(epochs), int(batch),
                                  ctypes.c_float(lr), int(seed), _ptr(hist)), self._h)
        return hist

    def lpc_loss_grad(self, geom, mb, params=None):
        """Mean loss and its gradient over the given configurations (params:
        None keeps the current ones)."""
        geom, mb = (np.ascontiguousarray(a, dtype=np.float32) for a in (geom, mb))
        pp = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        grad = np.zeros(int(lib().ibg_lpc_num_params()), np.float32)
        loss = ctypes.c_float()
        check(lib().ibg_lpc_loss_grad(self._h, int(mb.shape[0]), _ptr(geom), _ptr(mb), _ptr(pp),
                                      ctypes.byref(loss), _ptr(grad)), self._h)
        return loss.value, grad

    def lpc_apply(self, k: int, r):
        """The preconditioner action z = P_k r at the current body configuration
        (BF16 inference) and the geometry features it used [npts, 4]."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        geom = np.zeros((self.npoints, 4), np.float32)
        check(lib().ibg_lpc_apply(self._h, int(k), _ptr(r), _ptr(z), _ptr(geom)), self._h)
        return z, geom

    def beta(self, k: int) -> float:
        """Sub-step factor beta_k of M_k = beta_k C A_k^-1 B."""
        b = ctypes.c_double()
        check(lib().ibg_substep_beta(self._h, int(k), ctypes.byref(b)), self._h)
        return b.value

    def lpc_params(self) -> np.ndarray:
        p = np.zeros(int(lib().ibg_lpc_num_params()), np.float32)
        check(lib().ibg_lpc_get_params(self._h, _ptr(p), p.size), self._h)
        return p

    def lpc_set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        check(lib().ibg_lpc_set_params(self._h, _ptr(p), p.size), self._h)

    # -- operators (host buffers) ------------------------------------------
    def _op(self, name, *args, out_shape):
        out = np.zeros(out_shape)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if isinstance(a, np.ndarray) else a for a in args]
        cargs = [_ptr(a) if isinstance(a, np.ndarray) else a for a in arrs]
        check(getattr(lib(), name)(self._h, *cargs, _ptr(out)), self._h)
        return out

    def poisson(self, f):
        return self._op("ibg_poisson_solve", f, out_shape=self.grid.scalar().shape)

    def helmholtz(self, alpha, f):
        return self._op("ibg_helmholtz_solve", ctypes.c_double(alpha), f, out_shape=self.grid.scalar().shape)

    def nonlinear(self, q, w):
        return self._op("ibg_nonlinear", q, w, out_shape=self.grid.scalar().shape)

    def laplacian(self, f):
        return self._op("ibg_laplacian", f, out_shape=self.grid.scalar().shape)

    def model_B(self, f):
        return self._op("ibg_model_B", f, out_shape=self.grid.scalar().shape)

    def model_C(self, w):
        return self._op("ibg_model_C", w, out_shape=(2 * self.npoints,))

    def reg_to_boundary(self, q0):
        return self._op("ibg_reg_to_boundary", q0, out_shape=(2 * self.npoints,))

    def reg_to_flux(self, f):
        """Regularizer::toFlux: the Flux (every level) of a boundary vector."""
        return self._op("ibg_reg_to_flux", f, out_shape=self.grid.flux().shape)

    def projection_solve(self, k, a, b, f0):
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        f = np.ascontiguousarray(f0, dtype=np.float64).copy()
        w = np.zeros(self.grid.scalar().shape)
        check(lib().ibg_projection_solve(self._h, int(k), _ptr(a), _ptr(b), _ptr(w), _ptr(f)), self._h)
        return w, f


def autotune_log():
    """Launch shapes the autotuner chose in this process: one dict per
    (precision, pass, FFT length, lines, levels)."""
    n = lib().ibg_autotune_log(None, 0)
    buf = np.zeros(8 * max(n, 1), np.int32)
    n = lib().ibg_autotune_log(buf.ctypes.data_as(ctypes.c_void_p), n)
    keys = ("bytes", "pass", "fft_length", "lines", "levels", "pairs_per_cta", "threads", "twiddles_in_smem")
    return [dict(zip(keys, (int(v) for v in buf[8 * k:8 * k + 8]))) for k in range(n)]


def dst_form_log():
    """The autotuner's FFT-vs-GEMM choice for the FP32 DST passes in this process: one dict per
    grid shape timed."""
    n = lib().ibg_dst_form_log(None, 0)
    buf = np.zeros(6 * max(n, 1))
    n = lib().ibg_dst_form_log(buf.ctypes.data_as(ctypes.c_void_p), n)
    keys = ("nx", "ny", "levels", "gemm", "fft_us", "gemm_us")
    return [dict(zip(keys, (float(v) for v in buf[6 * k:6 * k + 6]))) for k in range(n)]


def sweep_form_log():
    """The autotuner's choice between the sweep's edge maps and its per-step line FFTs in this process:
    one dict per grid shape and precision timed."""
    n = lib().ibg_sweep_form_log(None, 0)
    buf = np.zeros(7 * max(n, 1))
    n = lib().ibg_sweep_form_log(buf.ctypes.data_as(ctypes.c_void_p), n)
    keys = ("nx", "ny", "levels", "bytes", "edge_maps", "edge_maps_us", "line_ffts_us")
    return [dict(zip(keys, (float(v) for v in buf[7 * k:7 * k + 7]))) for k in range(n)]


def pass_form_log():
    """The autotuner's choice of the FP64 DST passes' form (half length or odd extension) in this
    process: one dict per grid shape timed."""
    n = lib().ibg_pass_form_log(None, 0)
    buf = np.zeros(6 * max(n, 1))
    n = lib().ibg_pass_form_log(buf.ctypes.data_as(ctypes.c_void_p), n)
    keys = ("nx", "ny", "levels", "half_length", "half_length_us", "odd_extension_us")
    return [dict(zip(keys, (float(v) for v in buf[6 * k:6 * k + 6]))) for k in range(n)]


def from_workload(wl, precision: str = "fp64", stream=None, device: int = -1, precond: str = "none",
                  pc_refresh: int = 10, cg_graph: bool = True, pc_fallback_iter: int = 0):
    """Grid, model, solver and initial State for an ibpm_b200.configs.Workload."""
    grid = Grid(wl.nx, wl.ny, wl.ngrid, wl.length, wl.xoffset, wl.yoffset)
    geo = _geometry.parse(wl.geom)
    model = NavierStokesModel(grid, geo, wl.Re)
    solver = NonlinearIBSolver(grid, model, wl.dt, wl.scheme, wl.tol, precision=precision, stream=stream,
                               device=device, precond=precond, pc_refresh=pc_refresh, cg_graph=cg_graph,
                               pc_fallback_iter=pc_fallback_iter)
    x = State(grid, geo.num_points)
    w0 = wl.initial_vorticity()
    if w0 is not None:
        x.omega = w0
    return grid, model, solver, x


class Ensemble:
    """Independent simulations advanced together: one CUDA graph whose branches
    are the members' time steps (fixed bodies; each member keeps its own grid,
    Reynolds number, time step and bodies)."""

    def __init__(self, members):
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m.handle.value for m in self.members])
        h = ctypes.c_void_p()
        st = lib().ibg_ensemble_create(len(self.members), arr, ctypes.byref(h))
        if st < 0:
            raise IbgError(f"ibg_ensemble_create: {lib().ibg_ensemble_last_error(None).decode()}")
        self._h = h

    def advance(self, nsteps: int = 1):
        st = lib().ibg_ensemble_advance(self._h, int(nsteps))
        if st < 0:
            raise IbgError(f"ibg_ensemble_advance: {lib().ibg_ensemble_last_error(self._h).decode()}")

    def stream(self) -> int:
        return lib().ibg_ensemble_stream(self._h) or 0

    def set_shapes(self, pairs_per_cta: int = 0, threads: int = 128, edge_maps: bool = False):
        """One DST launch shape for all members (0 pairs: the rule); recaptured at the next advance."""
        st = lib().ibg_ensemble_set_shapes(self._h, int(pairs_per_cta), int(threads), int(edge_maps))
        if st < 0:
            raise IbgError(f"ibg_ensemble_set_shapes: {lib().ibg_ensemble_last_error(self._h).decode()}")

    def launches_per_step(self) -> int:
        return int(lib().ibg_ensemble_launches_per_step(self._h))

    def advance_host(self, states, nsteps: int = 1):
        """IBSolver::advance(State&) for every member: states[i] holds member i's State arrays omega, q, f
        (C-contiguous float64 in page-locked host memory, e.g. numpy views of pinned torch tensors).
        Each step copies every State in, advances and copies it back out, in one graph launch, so
        that one member's copies overlap the other members' steps."""
        n = len(self.members)
        if len(states) != n:
            raise ValueError("advance_host: one State per member")
        for x in states:
            for a in (x.omega, x.q, x.f):
                if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
                    raise ValueError("advance_host: State arrays must be C-contiguous float64")
        ptrs = [(ctypes.c_void_p * n)(*[getattr(x, k).ctypes.data for x in states]) for k in ("omega", "q", "f")]
        st = lib().ibg_ensemble_advance_host(self._h, int(nsteps), *ptrs)
        if st < 0:
            raise IbgError(f"ibg_ensemble_advance_host: {lib().ibg_ensemble_last_error(self._h).decode()}")

    def autotune(self, steps_per_trial: int = 3):
        """Choose each grid class's DST launch shape by timing ensemble steps (the trials advance every
        member); returns one dict per class."""
        rows = np.zeros(5 * max(1, len(self.members)), dtype=np.int32)
        n = lib().ibg_ensemble_autotune(self._h, int(steps_per_trial), rows.ctypes.data_as(ctypes.c_void_p),
                                        len(self.members))
        if n < 0:
            raise IbgError(f"ibg_ensemble_autotune: {lib().ibg_ensemble_last_error(self._h).decode()}")
        keys = ("nx", "ny", "us_per_step", "pairs_per_cta", "threads")
        return [dict(zip(keys, (int(v) for v in rows[5 * k:5 * k + 5]))) for k in range(n)]

    def host_launches_per_step(self) -> int:
        return int(lib().ibg_ensemble_host_launches_per_step(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().ibg_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
