"""CPU restatement of the IBPM time step (FP64, numpy).

TEST INFRASTRUCTURE ONLY.  This module is the parity checker for the CUDA
implementation in ``ibpm_b200``: only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg may import it.  The product path never
calls into it.

Parity is pinned: every operator here is checked against the reference
library itself (compiled from the reference sources with a project-written
FFTW shim into ``oracle/_ref/``; see ``oracle/Makefile``) and against the
golden fixtures in ``tests/golden/`` that were generated from it.

Layouts are the reference's (all citations are paths inside the reference
project):

* Scalar: ``(..., L, nx-1, ny-1)``, node (i, j) stored at ``[i-1, j-1]``
  (src/Scalar.h:76-90, src/Scalar.cc:81-89).
* Flux: ``(..., L, F1)`` with x-fluxes first (i in 0..nx, j in 0..ny-1,
  index i*ny + j) then y-fluxes at offset (nx+1)*ny (i in 0..nx-1,
  j in 0..ny, index i*(ny+1) + j) (src/Flux.h:176-185).
* BoundaryVector: ``[fx_0..fx_{n-1}, fy_0..fy_{n-1}]`` (src/BoundaryVector.h:65-69).

Leading batch dimensions (``...``) are supported by the elliptic solvers and
stencils so that the Cholesky matrix can be built for all basis vectors at once.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# ----------------------------------------------------------------------------
# Grid (src/Grid.h:89-128, src/Grid.cc:64-140)
# ----------------------------------------------------------------------------


@dataclass
class Grid:
    nx: int
    ny: int
    ngrid: int
    length: float
    xoffset: float
    yoffset: float
    xshift: float = 0.0
    yshift: float = 0.0

    def __post_init__(self):
        # src/Grid.cc:72 asserts multiples of 4 in debug builds only; the release build
        # (-DNDEBUG) nests with integer division, restated here for even sizes
        if self.ngrid > 1 and (self.nx % 2 or self.ny % 2):
            raise ValueError("nx and ny must be even when ngrid > 1")

    @property
    def dx(self) -> float:
        return self.length / self.nx

    def dx_lev(self, lev: int) -> float:
        return self.dx * (1 << lev)

    @property
    def nxext(self) -> int:  # src/Grid.h:60-62
        return int(math.floor(self.nx // 4 * (1 - self.xshift) + 0.5))

    @property
    def nyext(self) -> int:
        return int(math.floor(self.ny // 4 * (1 - self.yshift) + 0.5))

    def x_offset(self, lev: int) -> float:  # src/Grid.cc:104-106
        return self.xoffset + 0.5 * (self.xshift - 1) * ((1 << lev) - 1) * (self.nx * self.dx)

    def y_offset(self, lev: int) -> float:
        return self.yoffset + 0.5 * (self.yshift - 1) * ((1 << lev) - 1) * (self.ny * self.dx)

    @property
    def n_nodes(self) -> int:
        return (self.nx - 1) * (self.ny - 1)

    @property
    def n_xflux(self) -> int:
        return (self.nx + 1) * self.ny

    @property
    def n_flux(self) -> int:
        return 2 * self.nx * self.ny + self.nx + self.ny

    def scalar(self, batch=()) -> np.ndarray:
        return np.zeros(tuple(batch) + (self.ngrid, self.nx - 1, self.ny - 1))

    def flux(self, batch=()) -> np.ndarray:
        return np.zeros(tuple(batch) + (self.ngrid, self.n_flux))


# --- views -------------------------------------------------------------------


def _xf(g: Grid, q: np.ndarray, lev: int) -> np.ndarray:
    """x-flux view [i, j], i in 0..nx, j in 0..ny-1 (src/Flux.h:176-185)."""
    return q[..., lev, : g.n_xflux].reshape(q.shape[:-2] + (g.nx + 1, g.ny))


def _yf(g: Grid, q: np.ndarray, lev: int) -> np.ndarray:
    """y-flux view [i, j], i in 0..nx-1, j in 0..ny."""
    return q[..., lev, g.n_xflux:].reshape(q.shape[:-2] + (g.nx, g.ny + 1))


def _padded(g: Grid, s: np.ndarray, lev: int, fill=0.0) -> np.ndarray:
    """Level `lev` of a Scalar as a (nx+1, ny+1) node array; border = fill."""
    out = np.full(s.shape[:-3] + (g.nx + 1, g.ny + 1), fill, dtype=s.dtype)
    out[..., 1:-1, 1:-1] = s[..., lev, :, :]
    return out


# ----------------------------------------------------------------------------
# coarsify and getBC (src/Scalar.cc:46-64, :91-127)
# ----------------------------------------------------------------------------


def coarsify(g: Grid, s: np.ndarray) -> np.ndarray:
    """Full-weighting restriction of each finer level onto the overlap interior
    of the next coarser level, finest first (src/Scalar.cc:46-64)."""
    s = s.copy()
    nx, ny, nxe, nye = g.nx, g.ny, g.nxext, g.nyext
    for lev in range(1, g.ngrid):
        f = _padded(g, s, lev - 1)
        # coarse i in (nxe, nx/2+nxe) -> fine ii = 2(i-nxe) in [2, nx-2], step 2
        c = (0.25 * f[..., 2:nx - 1:2, 2:ny - 1:2]
             + 0.125 * (f[..., 3:nx:2, 2:ny - 1:2] + f[..., 2:nx - 1:2, 3:ny:2]
                        + f[..., 1:nx - 2:2, 2:ny - 1:2] + f[..., 2:nx - 1:2, 1:ny - 2:2])
             + 0.0625 * (f[..., 3:nx:2, 3:ny:2] + f[..., 3:nx:2, 1:ny - 2:2]
                         + f[..., 1:nx - 2:2, 3:ny:2] + f[..., 1:nx - 2:2, 1:ny - 2:2]))
        s[..., lev, nxe:nxe + nx // 2 - 1, nye:nye + ny // 2 - 1] = c
    return s


@dataclass
class BC:
    """Boundary ring values: bottom/top indexed by i in 0..nx, left/right by j in 0..ny."""
    bottom: np.ndarray
    top: np.ndarray
    left: np.ndarray
    right: np.ndarray


def get_bc(g: Grid, s: np.ndarray, lev: int) -> BC:
    """Boundary values of level `lev` from level lev+1: coincident nodes are
    copied, in-between nodes averaged (src/Scalar.cc:91-127)."""
    nx, ny, nxe, nye = g.nx, g.ny, g.nxext, g.nyext
    c = _padded(g, s, lev + 1)
    i = np.arange(nx + 1)
    ii = i // 2 + nxe
    odd_i = (i % 2 == 1)
    j = np.arange(ny + 1)
    jj = j // 2 + nye
    odd_j = (j % 2 == 1)

    def row(jc):
        a = c[..., ii, jc]
        b = c[..., np.minimum(ii + 1, nx), jc]
        return np.where(odd_i, 0.5 * (a + b), a)

    def col(ic):
        a = c[..., ic, jj]
        b = c[..., ic, np.minimum(jj + 1, ny)]
        return np.where(odd_j, 0.5 * (a + b), a)

    return BC(bottom=row(nye), top=row(ny // 2 + nye), left=col(nxe), right=col(nx // 2 + nxe))


def zero_bc(g: Grid, batch=()) -> BC:
    z = lambda n: np.zeros(tuple(batch) + (n,))
    return BC(z(g.nx + 1), z(g.nx + 1), z(g.ny + 1), z(g.ny + 1))


def bc_ring(g: Grid, bc: BC) -> np.ndarray:
    """Pack a BC into the reference's 1-D ring order (src/BC.h:22-96)."""
    nx, ny = g.nx, g.ny
    ring = np.zeros(bc.left.shape[:-1] + (2 * (nx + ny),))
    ring[..., 0:ny + 1] = bc.left
    ring[..., ny:ny + nx + 1] = bc.top
    for jv in range(ny, -1, -1):
        ring[..., 2 * ny + nx - jv] = bc.right[..., jv]
    for iv in range(nx, 0, -1):
        ring[..., 2 * (nx + ny) - iv] = bc.bottom[..., iv]
    return ring


def _with_bc(g: Grid, s: np.ndarray, lev: int, bc: BC) -> np.ndarray:
    p = _padded(g, s, lev)
    p[..., :, 0] = bc.bottom
    p[..., :, g.ny] = bc.top
    p[..., 0, :] = bc.left
    p[..., g.nx, :] = bc.right
    return p


def _level_bc(g: Grid, s: np.ndarray, lev: int) -> BC:
    if lev == g.ngrid - 1:
        return zero_bc(g, s.shape[:-3])
    return get_bc(g, s, lev)


# ----------------------------------------------------------------------------
# Curl, Laplacian (src/VectorOperations.cc:33-146)
# ----------------------------------------------------------------------------


def curl_flux(g: Grid, q: np.ndarray) -> np.ndarray:
    """Scalar = curl of a Flux, level by level (src/VectorOperations.cc:33-54)."""
    out = g.scalar(q.shape[:-2])
    for lev in range(g.ngrid):
        dx = g.dx_lev(lev)
        bydx2 = 1.0 / (dx * dx)
        qx, qy = _xf(g, q, lev), _yf(g, q, lev)
        out[..., lev, :, :] = (qy[..., 1:, 1:-1] - qy[..., :-1, 1:-1]
                               + qx[..., 1:-1, :-1] - qx[..., 1:-1, 1:]) * bydx2
    return out


def curl_scalar(g: Grid, f: np.ndarray) -> np.ndarray:
    """Flux = curl of a Scalar, coarsest level first, boundary values from the
    next coarser level (src/VectorOperations.cc:63-123)."""
    q = g.flux(f.shape[:-3])
    nx, ny = g.nx, g.ny
    for lev in range(g.ngrid - 1, -1, -1):
        bc = _level_bc(g, f, lev)
        p = _with_bc(g, f, lev, bc)
        qx, qy = _xf(g, q, lev), _yf(g, q, lev)
        # x-fluxes: interior i in 1..nx-1, all j in 0..ny-1: u = f(i,j+1) - f(i,j)
        qx[..., 1:nx, :] = p[..., 1:nx, 1:] - p[..., 1:nx, :-1]
        # left/right boundaries
        qx[..., 0, :] = bc.left[..., 1:] - bc.left[..., :-1]
        qx[..., nx, :] = bc.right[..., 1:] - bc.right[..., :-1]
        # y-fluxes: all i in 0..nx-1, interior j in 1..ny-1: v = f(i,j) - f(i+1,j)
        qy[..., :, 1:ny] = p[..., :-1, 1:ny] - p[..., 1:, 1:ny]
        qy[..., :, 0] = bc.bottom[..., :-1] - bc.bottom[..., 1:]
        qy[..., :, ny] = bc.top[..., :-1] - bc.top[..., 1:]
        _xf_set(g, q, lev, qx)
        _yf_set(g, q, lev, qy)
    return q


def _xf_set(g, q, lev, qx):
    q[..., lev, : g.n_xflux] = qx.reshape(qx.shape[:-2] + (-1,))


def _yf_set(g, q, lev, qy):
    q[..., lev, g.n_xflux:] = qy.reshape(qy.shape[:-2] + (-1,))


def laplacian(g: Grid, f: np.ndarray) -> np.ndarray:
    """L f = -Curl(Curl(f)) (src/VectorOperations.cc:133-146)."""
    return -curl_flux(g, curl_scalar(g, f))


# ----------------------------------------------------------------------------
# flux <-> node velocity with multi-domain interface stencils
# (src/VectorOperations.cc:488-916)
# ----------------------------------------------------------------------------


def flux_to_xvel(g: Grid, q: np.ndarray) -> np.ndarray:
    """u at nodes from x-fluxes; coarse overlap interior is left NaN
    (uninitialised in the reference) (src/VectorOperations.cc:488-576)."""
    nx, ny, nx2, ny2 = g.nx, g.ny, g.nxext, g.nyext
    u = np.full(q.shape[:-2] + (g.ngrid, nx + 1, ny + 1), np.nan)
    qx0 = _xf(g, q, 0)
    o2d = 1.0 / (2 * g.dx)
    u[..., 0, 1:nx, 1:ny] = (qx0[..., 1:nx, 1:ny] + qx0[..., 1:nx, 0:ny - 1]) * o2d
    for lev in range(1, g.ngrid):
        bydx = 1.0 / g.dx_lev(lev)
        qx, qf = _xf(g, q, lev), _xf(g, q, lev - 1)

        def avg(isl, jsl):
            i0, i1 = isl
            j0, j1 = jsl
            return (qx[..., i0:i1, j0:j1] + qx[..., i0:i1, j0 - 1:j1 - 1]) * 0.5 * bydx

        # B: left and right borders
        u[..., lev, 1:nx2, 1:ny] = avg((1, nx2), (1, ny))
        u[..., lev, nx // 2 + nx2 + 1:nx, 1:ny] = avg((nx // 2 + nx2 + 1, nx), (1, ny))
        # C: top and bottom borders
        u[..., lev, nx2:nx // 2 + nx2 + 1, 1:ny2] = avg((nx2, nx // 2 + nx2 + 1), (1, ny2))
        u[..., lev, nx2:nx // 2 + nx2 + 1, ny // 2 + ny2 + 1:ny] = avg(
            (nx2, nx // 2 + nx2 + 1), (ny // 2 + ny2 + 1, ny))
        # D: left/right interfaces excluding corners
        for ic in (nx2, nx // 2 + nx2):
            u[..., lev, ic, ny2 + 1:ny // 2 + ny2] = avg((ic, ic + 1), (ny2 + 1, ny // 2 + ny2))[..., 0, :]
        # E: top/bottom interfaces excluding corners
        i = np.arange(nx2 + 1, nx // 2 + nx2)
        ii = 2 * (i - nx2)
        u[..., lev, i, ny2] = (qx[..., i, ny2 - 1] * 2. / 3 + qf[..., ii, 0] * 1. / 3
                               + (qf[..., ii - 1, 0] + qf[..., ii + 1, 0]) * 1. / 6) * bydx
        jt = ny // 2 + ny2
        u[..., lev, i, jt] = (qx[..., i, jt] * 2. / 3 + qf[..., ii, ny - 1] * 1. / 3
                              + (qf[..., ii - 1, ny - 1] + qf[..., ii + 1, ny - 1]) * 1. / 6) * bydx
        # F: corners
        il, ir = nx2, nx // 2 + nx2
        jb, jt = ny2, ny // 2 + ny2
        u[..., lev, il, jb] = (qx[..., il, jb - 1] * 8. / 15 + qx[..., il, jb] * 6. / 15
                               + qf[..., 1, 0] * 2. / 15) * bydx
        u[..., lev, ir, jb] = (qx[..., ir, jb - 1] * 8. / 15 + qx[..., ir, jb] * 6. / 15
                               + qf[..., nx - 1, 0] * 2. / 15) * bydx
        u[..., lev, il, jt] = (qx[..., il, jt] * 8. / 15 + qx[..., il, jt - 1] * 6. / 15
                               + qf[..., 1, ny - 1] * 2. / 15) * bydx
        u[..., lev, ir, jt] = (qx[..., ir, jt] * 8. / 15 + qx[..., ir, jt - 1] * 6. / 15
                               + qf[..., nx - 1, ny - 1] * 2. / 15) * bydx
    return u[..., 1:nx, 1:ny]


def flux_to_yvel(g: Grid, q: np.ndarray) -> np.ndarray:
    """v at nodes from y-fluxes (src/VectorOperations.cc:578-667)."""
    nx, ny, nx2, ny2 = g.nx, g.ny, g.nxext, g.nyext
    v = np.full(q.shape[:-2] + (g.ngrid, nx + 1, ny + 1), np.nan)
    qy0 = _yf(g, q, 0)
    o2d = 1.0 / (2 * g.dx)
    v[..., 0, 1:nx, 1:ny] = (qy0[..., 0:nx - 1, 1:ny] + qy0[..., 1:nx, 1:ny]) * o2d
    for lev in range(1, g.ngrid):
        bydx = 1.0 / g.dx_lev(lev)
        qy, qf = _yf(g, q, lev), _yf(g, q, lev - 1)

        def avg(isl, jsl):
            i0, i1 = isl
            j0, j1 = jsl
            return (qy[..., i0:i1, j0:j1] + qy[..., i0 - 1:i1 - 1, j0:j1]) * 0.5 * bydx

        # B: top and bottom borders
        v[..., lev, 1:nx, 1:ny2] = avg((1, nx), (1, ny2))
        v[..., lev, 1:nx, ny // 2 + ny2 + 1:ny] = avg((1, nx), (ny // 2 + ny2 + 1, ny))
        # C: left and right borders
        v[..., lev, 1:nx2, ny2:ny // 2 + ny2 + 1] = avg((1, nx2), (ny2, ny // 2 + ny2 + 1))
        v[..., lev, nx // 2 + nx2 + 1:nx, ny2:ny // 2 + ny2 + 1] = avg(
            (nx // 2 + nx2 + 1, nx), (ny2, ny // 2 + ny2 + 1))
        # D: top/bottom interfaces excluding corners
        for jc in (ny2, ny // 2 + ny2):
            v[..., lev, nx2 + 1:nx // 2 + nx2, jc] = avg((nx2 + 1, nx // 2 + nx2), (jc, jc + 1))[..., :, 0]
        # E: left/right interfaces excluding corners
        j = np.arange(ny2 + 1, ny // 2 + ny2)
        jj = 2 * (j - ny2)
        v[..., lev, nx2, j] = (qy[..., nx2 - 1, j] * 2. / 3 + qf[..., 0, jj] * 1. / 3
                               + (qf[..., 0, jj - 1] + qf[..., 0, jj + 1]) * 1. / 6) * bydx
        ir = nx // 2 + nx2
        v[..., lev, ir, j] = (qy[..., ir, j] * 2. / 3 + qf[..., nx - 1, jj] * 1. / 3
                              + (qf[..., nx - 1, jj - 1] + qf[..., nx - 1, jj + 1]) * 1. / 6) * bydx
        # F: corners
        il, ir = nx2, nx // 2 + nx2
        jb, jt = ny2, ny // 2 + ny2
        v[..., lev, il, jb] = (qy[..., il - 1, jb] * 8. / 15 + qy[..., il, jb] * 6. / 15
                               + qf[..., 0, 1] * 2. / 15) * bydx
        v[..., lev, il, jt] = (qy[..., il - 1, jt] * 8. / 15 + qy[..., il, jt] * 6. / 15
                               + qf[..., 0, ny - 1] * 2. / 15) * bydx
        v[..., lev, ir, jb] = (qy[..., ir, jb] * 8. / 15 + qy[..., ir - 1, jb] * 6. / 15
                               + qf[..., nx - 1, 1] * 2. / 15) * bydx
        v[..., lev, ir, jt] = (qy[..., ir, jt] * 8. / 15 + qy[..., ir - 1, jt] * 6. / 15
                               + qf[..., nx - 1, ny - 1] * 2. / 15) * bydx
    return v[..., 1:nx, 1:ny]


def xvel_to_flux(g: Grid, u: np.ndarray, q: np.ndarray) -> None:
    """x-fluxes from node values u (in place on q); reads only defined nodes
    of u (src/VectorOperations.cc:669-786)."""
    nx, ny, nx2, ny2 = g.nx, g.ny, g.nxext, g.nyext
    L = g.ngrid
    P = [_padded(g, u, lev) for lev in range(L)]
    for lev in range(L):
        dx = g.dx_lev(lev)
        qx = _xf(g, q, lev).copy()
        p = P[lev]

        def avg(i0, i1, j0, j1):
            return (p[..., i0:i1, j0:j1] + p[..., i0:i1, j0 + 1:j1 + 1]) * 0.5 * dx

        if lev == 0:
            qx[..., 1:nx, 1:ny - 1] = avg(1, nx, 1, ny - 1)
        else:
            # B
            qx[..., 1:nx, 1:ny2] = avg(1, nx, 1, ny2)
            qx[..., 1:nx, ny // 2 + ny2:ny - 1] = avg(1, nx, ny // 2 + ny2, ny - 1)
            # D
            qx[..., 1:nx2 + 1, ny2:ny // 2 + ny2] = avg(1, nx2 + 1, ny2, ny // 2 + ny2)
            qx[..., nx // 2 + nx2:nx, ny2:ny // 2 + ny2] = avg(nx // 2 + nx2, nx, ny2, ny // 2 + ny2)
            # G: injection from the finer level's fluxes (already final)
            qf = _xf(g, q, lev - 1)
            i = np.arange(nx2 + 1, nx // 2 + nx2)
            j = np.arange(ny2, ny // 2 + ny2)
            ii = (2 * (i - nx2))[:, None]
            jj = (2 * (j - ny2))[None, :]
            qx[..., nx2 + 1:nx // 2 + nx2, ny2:ny // 2 + ny2] = qf[..., ii, jj] + qf[..., ii, jj + 1]
        # A: left/right boundaries
        if lev == L - 1:
            qx[..., 0, :] = 0.0
            qx[..., nx, :] = 0.0
        else:
            c = P[lev + 1]
            jeven = np.arange(0, ny - 1, 2)
            jj = jeven // 2 + ny2
            for ic, ib in ((nx2, 0), (nx // 2 + nx2, nx)):
                qx[..., ib, jeven] = (0.75 * c[..., ic, jj] + 0.25 * c[..., ic, jj + 1]) * dx
                qx[..., ib, jeven + 1] = (0.25 * c[..., ic, jj] + 0.75 * c[..., ic, jj + 1]) * dx
        # C: bottom/top rows
        if lev == L - 1:
            qx[..., 1:nx, 0] = p[..., 1:nx, 1] * 0.5 * dx
            qx[..., 1:nx, ny - 1] = p[..., 1:nx, ny - 1] * 0.5 * dx
        else:
            c = P[lev + 1]
            ie = np.arange(2, nx, 2)
            iic = ie // 2 + nx2
            qx[..., ie, 0] = (p[..., ie, 1] + c[..., iic, ny2]) * 0.5 * dx
            qx[..., ie, ny - 1] = (p[..., ie, ny - 1] + c[..., iic, ny // 2 + ny2]) * 0.5 * dx
            io = np.arange(1, nx, 2)
            iic = io // 2 + nx2
            qx[..., io, 0] = (0.5 * p[..., io, 1] + 0.25 * c[..., iic, ny2] + 0.25 * c[..., iic + 1, ny2]) * dx
            qx[..., io, ny - 1] = (0.5 * p[..., io, ny - 1] + 0.25 * c[..., iic, ny // 2 + ny2]
                                   + 0.25 * c[..., iic + 1, ny // 2 + ny2]) * dx
        _xf_set(g, q, lev, qx)


def yvel_to_flux(g: Grid, v: np.ndarray, q: np.ndarray) -> None:
    """y-fluxes from node values v (in place on q) (src/VectorOperations.cc:788-916)."""
    nx, ny, nx2, ny2 = g.nx, g.ny, g.nxext, g.nyext
    L = g.ngrid
    P = [_padded(g, v, lev) for lev in range(L)]
    for lev in range(L):
        dx = g.dx_lev(lev)
        qy = _yf(g, q, lev).copy()
        p = P[lev]

        def avg(i0, i1, j0, j1):
            return (p[..., i0:i1, j0:j1] + p[..., i0 + 1:i1 + 1, j0:j1]) * 0.5 * dx

        if lev == 0:
            qy[..., 1:nx - 1, 1:ny] = avg(1, nx - 1, 1, ny)
        else:
            # B
            qy[..., 1:nx2, 1:ny] = avg(1, nx2, 1, ny)
            qy[..., nx // 2 + nx2:nx - 1, 1:ny] = avg(nx // 2 + nx2, nx - 1, 1, ny)
            # D
            qy[..., nx2:nx // 2 + nx2, 1:ny2 + 1] = avg(nx2, nx // 2 + nx2, 1, ny2 + 1)
            qy[..., nx2:nx // 2 + nx2, ny // 2 + ny2:ny] = avg(nx2, nx // 2 + nx2, ny // 2 + ny2, ny)
            # G
            qf = _yf(g, q, lev - 1)
            i = np.arange(nx2, nx // 2 + nx2)
            j = np.arange(ny2 + 1, ny // 2 + ny2)
            ii = (2 * (i - nx2))[:, None]
            jj = (2 * (j - ny2))[None, :]
            qy[..., nx2:nx // 2 + nx2, ny2 + 1:ny // 2 + ny2] = qf[..., ii, jj] + qf[..., ii + 1, jj]
        # A: bottom/top boundaries
        if lev == L - 1:
            qy[..., :, 0] = 0.0
            qy[..., :, ny] = 0.0
        else:
            c = P[lev + 1]
            ieven = np.arange(0, nx - 1, 2)
            ii = ieven // 2 + nx2
            for jc, jb in ((ny2, 0), (ny // 2 + ny2, ny)):
                qy[..., ieven, jb] = (0.75 * c[..., ii, jc] + 0.25 * c[..., ii + 1, jc]) * dx
                qy[..., ieven + 1, jb] = (0.25 * c[..., ii, jc] + 0.75 * c[..., ii + 1, jc]) * dx
        # C: left/right columns
        if lev == L - 1:
            qy[..., 0, 1:ny] = p[..., 1, 1:ny] * 0.5 * dx
            qy[..., nx - 1, 1:ny] = p[..., nx - 1, 1:ny] * 0.5 * dx
        else:
            c = P[lev + 1]
            je = np.arange(2, ny, 2)
            jjc = je // 2 + ny2
            qy[..., 0, je] = (p[..., 1, je] + c[..., nx2, jjc]) * 0.5 * dx
            qy[..., nx - 1, je] = (p[..., nx - 1, je] + c[..., nx // 2 + nx2, jjc]) * 0.5 * dx
            jo = np.arange(1, ny, 2)
            jjc = jo // 2 + ny2
            qy[..., 0, jo] = (0.5 * p[..., 1, jo] + 0.25 * c[..., nx2, jjc] + 0.25 * c[..., nx2, jjc + 1]) * dx
            qy[..., nx - 1, jo] = (0.5 * p[..., nx - 1, jo] + 0.25 * c[..., nx // 2 + nx2, jjc]
                                   + 0.25 * c[..., nx // 2 + nx2, jjc + 1]) * dx
        _yf_set(g, q, lev, qy)


def cross_product(g: Grid, q: np.ndarray, w: np.ndarray) -> np.ndarray:
    """q x w = (w v, -w u) as a Flux (src/VectorOperations.cc:438-457)."""
    u = flux_to_xvel(g, q) * w * -1.0
    v = flux_to_yvel(g, q) * w
    out = g.flux(q.shape[:-2])
    xvel_to_flux(g, v, out)
    yvel_to_flux(g, u, out)
    return out


def nonlinear(g: Grid, q: np.ndarray, w: np.ndarray) -> np.ndarray:
    """NonlinearIBSolver::N = Curl(CrossProduct(q, omega)) (src/IBSolver.cc:205-209)."""
    return curl_flux(g, cross_product(g, q, w))


def cross_product_flux(g: Grid, q1: np.ndarray, q2: np.ndarray) -> np.ndarray:
    """CrossProduct(Flux, Flux) = u1 v2 - u2 v1 at the nodes, then coarsified over the
    overlap regions (src/VectorOperations.cc:465-486)."""
    f = flux_to_xvel(g, q1) * flux_to_yvel(g, q2)
    f = f - flux_to_xvel(g, q2) * flux_to_yvel(g, q1)
    return coarsify(g, f)


def adjoint(g: Grid, q: np.ndarray, w: np.ndarray, q0: np.ndarray, w0: np.ndarray) -> np.ndarray:
    """AdjointIBSolver::N = Laplacian(CrossProduct(q0, q)) - Curl(CrossProduct(q, omega0))
    (src/IBSolver.cc:218-222)."""
    return laplacian(g, cross_product_flux(g, q0, q)) - nonlinear(g, q, w0)


def linearized(g: Grid, q: np.ndarray, w: np.ndarray, q0: np.ndarray, w0: np.ndarray) -> np.ndarray:
    """LinearizedIBSolver::N = Curl(q0 x omega + q x omega0) (src/IBSolver.cc:211-216); the periodic
    form uses the base state of phase timestep % period (src/IBSolver.cc:224-232)."""
    v = cross_product(g, q0, w)
    v = v + cross_product(g, q, w0)
    return curl_flux(g, v)


# ----------------------------------------------------------------------------
# Elliptic solvers (src/EllipticSolver2d.cc:26-185, src/EllipticSolver.cc:47-108)
# ----------------------------------------------------------------------------


def dst1(x: np.ndarray, axis: int) -> np.ndarray:
    """Unnormalised DST-I (FFTW RODFT00): Y_k = 2 sum_j X_j sin(pi(j+1)(k+1)/(n+1)),
    read off the FFT of the odd extension of length 2(n+1)."""
    x = np.moveaxis(x, axis, -1)
    n = x.shape[-1]
    ext = np.zeros(x.shape[:-1] + (2 * (n + 1),))
    ext[..., 1:n + 1] = x
    ext[..., n + 2:] = -x[..., ::-1]
    y = -np.fft.fft(ext, axis=-1)[..., 1:n + 1].imag
    return np.moveaxis(y, -1, axis)


def laplacian_eigenvalues(nx: int, ny: int, dx: float) -> np.ndarray:
    """lambda_ij = 2 (cos(pi i/nx) + cos(pi j/ny) - 2)/dx^2 (src/EllipticSolver2d.cc:42-54)."""
    pi = 4.0 * math.atan(1.0)
    i = np.arange(1, nx)[:, None]
    j = np.arange(1, ny)[None, :]
    return 2.0 * (np.cos((pi * i) / nx) + np.cos((pi * j) / ny) - 2.0) * (1.0 / (dx * dx))


def eigen_inverse(kind: str, nx: int, ny: int, dx: float, alpha: float = 0.0) -> np.ndarray:
    lam = laplacian_eigenvalues(nx, ny, dx)
    if kind == "poisson":  # src/EllipticSolver2d.cc:115-122
        return 1.0 / lam
    return 1.0 / (1 + alpha * lam)  # src/EllipticSolver2d.cc:156-163


def solve2d(f: np.ndarray, eiginv: np.ndarray, nx: int, ny: int) -> np.ndarray:
    """Single-level solve with zero boundary values (src/EllipticSolver2d.cc:87-95)."""
    u = dst1(dst1(f, -2), -1) * eiginv
    u = dst1(dst1(u, -2), -1)
    return u * (1.0 / (2 * nx * 2 * ny))


def lift_bc(f: np.ndarray, bc: BC, c: float) -> np.ndarray:
    """rhs = f - c * bc on the first/last interior rows and columns
    (getRHS: src/EllipticSolver2d.cc:125-144 with c = 1/dx^2, :166-185 with c = alpha/dx^2)."""
    r = f.copy()
    r[..., :, 0] -= bc.bottom[..., 1:-1] * c
    r[..., :, -1] -= bc.top[..., 1:-1] * c
    r[..., 0, :] -= bc.left[..., 1:-1] * c
    r[..., -1, :] -= bc.right[..., 1:-1] * c
    return r


class EllipticSolver:
    """Multi-domain Poisson (kind='poisson') or Helmholtz (1 + alpha L) solver
    (src/EllipticSolver.cc:47-108)."""

    def __init__(self, g: Grid, kind: str, alpha: float = 0.0):
        self.g, self.kind, self.alpha = g, kind, alpha
        self.eig = [eigen_inverse(kind, g.nx, g.ny, g.dx_lev(l), alpha) for l in range(g.ngrid)]

    def solve(self, f: np.ndarray) -> np.ndarray:
        g = self.g
        rhs = coarsify(g, f)
        u = np.zeros_like(rhs)
        for lev in range(g.ngrid - 1, -1, -1):
            r = rhs[..., lev, :, :]
            if lev != g.ngrid - 1:
                dx = g.dx_lev(lev)
                c = (1.0 / (dx * dx)) if self.kind == "poisson" else (self.alpha / (dx * dx))
                r = lift_bc(r, get_bc(g, u, lev), c)
            u[..., lev, :, :] = solve2d(r, self.eig[lev], g.nx, g.ny)
        return u


# ----------------------------------------------------------------------------
# Regularizer (src/Regularizer.cc:31-128)
# ----------------------------------------------------------------------------


def delta_function(r: np.ndarray) -> np.ndarray:
    """Roma-Peskin-Berger 3-cell discrete delta (src/Regularizer.cc:39-49)."""
    r = np.asarray(r, dtype=float)
    out = np.zeros_like(r)
    a = r <= 0.5
    b = (r > 0.5) & (r <= 1.5)
    out[a] = (1 + np.sqrt(1 - 3 * r[a] * r[a])) / 3
    rb = r[b]
    out[b] = (5 - 3 * rb - np.sqrt(1 - 3 * (1 - rb) * (1 - rb))) / 6
    return out


class Regularizer:
    """Association list between boundary points and level-0 fluxes.

    The reference builds it by scanning every level-0 flux for every point
    (src/Regularizer.cc:54-90); here only the fluxes within two cells of each
    point are scanned, which yields the same list in the same order (dir,
    point, flux index)."""

    def __init__(self, g: Grid):
        self.g = g
        self.flux_idx = np.zeros(0, dtype=np.int64)
        self.bnd_idx = np.zeros(0, dtype=np.int64)
        self.weight = np.zeros(0)

    def update(self, xy: np.ndarray) -> None:
        g = self.g
        h = g.dx
        n = xy.shape[0]
        x0, y0 = g.x_offset(0), g.y_offset(0)
        fl, bl, wl = [], [], []
        for d in range(2):
            for p in range(n):
                px, py = xy[p, 0], xy[p, 1]
                if d == 0:   # x-flux (i, j) at (x0 + i h, y0 + (j + .5) h)
                    ni, nj, offx, offy, base, stride = g.nx + 1, g.ny, 0.0, 0.5, 0, g.ny
                else:        # y-flux (i, j) at (x0 + (i + .5) h, y0 + j h)
                    ni, nj, offx, offy, base, stride = g.nx, g.ny + 1, 0.5, 0.0, g.n_xflux, g.ny + 1
                ic = int(math.floor((px - x0) / h - offx))
                jc = int(math.floor((py - y0) / h - offy))
                i = np.arange(max(ic - 2, 0), min(ic + 4, ni))
                j = np.arange(max(jc - 2, 0), min(jc + 4, nj))
                if i.size == 0 or j.size == 0:
                    continue
                I, J = np.meshgrid(i, j, indexing="ij")
                fx = x0 + (I + offx) * h
                fy = y0 + (J + offy) * h
                dxn = np.abs(fx - px) / h
                dyn = np.abs(fy - py) / h
                m = (dxn < 1.5) & (dyn < 1.5)
                idx = base + I * stride + J
                order = np.argsort(idx[m], kind="stable")
                fl.append(idx[m][order])
                wl.append((delta_function(dxn[m]) * delta_function(dyn[m]))[order])
                bl.append(np.full(order.size, d * n + p))
        self.flux_idx = np.concatenate(fl) if fl else np.zeros(0, np.int64)
        self.bnd_idx = np.concatenate(bl) if bl else np.zeros(0, np.int64)
        self.weight = np.concatenate(wl) if wl else np.zeros(0)
        self.n_points = n

    def to_flux(self, f: np.ndarray) -> np.ndarray:
        """E^T: smear boundary values onto level-0 fluxes, times dx (src/Regularizer.cc:92-109)."""
        g = self.g
        q = g.flux(f.shape[:-1])
        acc = np.zeros(f.shape[:-1] + (g.n_flux,))
        contrib = self.weight * f[..., self.bnd_idx]
        if f.ndim == 1:
            np.add.at(acc, self.flux_idx, contrib)
        else:
            _batched_add(acc, self.flux_idx, contrib)
        q[..., 0, :] = acc * g.dx
        return q

    def to_boundary(self, q: np.ndarray) -> np.ndarray:
        """E: interpolate level-0 fluxes to boundary points, divided by dx (src/Regularizer.cc:111-128)."""
        g = self.g
        out = np.zeros(q.shape[:-2] + (2 * self.n_points,))
        contrib = self.weight * q[..., 0, self.flux_idx]
        if q.ndim == 2:
            np.add.at(out, self.bnd_idx, contrib)
        else:
            _batched_add(out, self.bnd_idx, contrib)
        return out / g.dx


def _batched_add(acc, idx, vals):
    flat = acc.reshape(-1, acc.shape[-1])
    v = vals.reshape(-1, vals.shape[-1])
    for b in range(flat.shape[0]):
        np.add.at(flat[b], idx, v[b])


# ----------------------------------------------------------------------------
# Bodies and kinematics (src/RigidBody.cc:105-131, :586-609; src/TangentSE2.h:83-107;
# the Motion subclasses named below)
# ----------------------------------------------------------------------------

MOTION_PARAMS = {"none": 0, "fixed": 3, "pitchplunge": 6, "fixedvel": 3, "sigmoidalstep": 3, "lagstep1": 4,
                 "lagstep2": 4, "eldredge": 6, "eldredgecombined2": 12, "eldredge1": 6, "eldredge2": 6,
                 "motionfile": 0, "motionfileperiodic": 1}


def _eld_G(a, t1, t2, t3, t4, t):
    """G(t) of Eldredge's smoothed ramp (src/EldredgeManeuver.h:56-57)."""
    return math.log((math.cosh(a * (t - t1)) * math.cosh(a * (t - t4))) /
                    (math.cosh(a * (t - t2)) * math.cosh(a * (t - t3))))


def _eld_dG(a, t1, t2, t3, t4, t):
    return a * (math.tanh(a * (t - t1)) - math.tanh(a * (t - t2)) - math.tanh(a * (t - t3)) + math.tanh(a * (t - t4)))


def _eld_max(a, a4, t1, t2, t3, t4):
    """maxG = G((t2 + t3)/2) (src/EldredgeManeuver.h:42-43); EldredgeCombined2 uses `a` in the t4 factor of its
    pitch ramp (src/EldredgeCombined2.h:59), hence the separate a4."""
    tt = (t2 + t3) / 2.0
    return math.log((math.cosh(a * (tt - t1)) * math.cosh(a4 * (tt - t4))) /
                    (math.cosh(a * (tt - t2)) * math.cosh(a * (tt - t3))))


@dataclass
class Body:
    ref_xy: np.ndarray                 # (n, 2) reference points
    center: tuple = (0.0, 0.0)
    motion: str = "none"               # a key of MOTION_PARAMS
    params: tuple = ()                 # the geometry file's numbers, in order
    table: np.ndarray = None           # motion file rows (t, x, y, theta, xdot, ydot, thetadot)
    # running integrals of FixedVelocity / Eldredge2 / EldredgeCombined2 (fresh Motion object)
    hist: dict = field(default_factory=lambda: {"x": 0.0, "y": 0.0, "th": 0.0, "g": 0.0, "told": 0.0})

    @property
    def stationary(self) -> bool:
        return self.motion in ("none", "fixed")

    def transformation(self, t: float):
        """Motion::getTransformation(t): (x, y, theta, xdot, ydot, thetadot) of the body frame.  The
        stateful motions advance their history, as the reference's mutable members do."""
        pi = 4.0 * math.atan(1.0)
        m, p, h = self.motion, self.params, self.hist
        if m == "pitchplunge":  # src/PitchPlunge.h:30-58
            twopi = 8.0 * math.atan(1.0)
            ap, fp, php, ay, fy, phy = p
            fp, fy = fp * twopi, fy * twopi
            y = ay * math.sin(fy * t + phy)
            ydot = ay * fy * math.cos(fy * t + phy)
            th = ap * math.sin(fp * t + php)
            thdot = ap * fp * math.cos(fp * t + php)
            return (0.0, y, th, 0.0, ydot, thdot)
        if m == "fixed":  # src/FixedPosition.h:42-44
            x, y, th = p
            return (x, y, th, 0.0, 0.0, 0.0)
        if m == "fixedvel":  # src/FixedVelocity.h:42-50
            dtt = t - h["told"]
            if dtt > 1:
                dtt = 0.0
            h["x"] += p[0] * dtt
            h["y"] += p[1] * dtt
            h["th"] += p[2] * dtt
            h["told"] = t
            return (h["x"], h["y"], h["th"], p[0], p[1], p[2])
        if m == "sigmoidalstep":  # src/SigmoidalStep.h:41-51
            amp, dur, t0 = p
            arg = 12.0 * (t - t0) / dur - 6.0
            coeff = 12.0 / (dur * math.sqrt(pi))
            return (0.0, 0.0, 0.5 * amp * (pi / 180) * (1.0 + math.erf(arg)), 0.0, 0.0,
                    amp * (pi / 180) * coeff * math.exp(-arg * arg))
        if m in ("lagstep1", "lagstep2"):  # src/LagStep1.h:41-62, src/LagStep2.h:41-62
            amp, pw, tau, t0 = p
            td = t - t0
            ampr = amp * (pi / 180)
            if td <= 0:
                a = ad = 0.0
            elif td <= pw:
                if m == "lagstep1":
                    a, ad = td + tau * math.exp(-td / tau) - tau, 1 - math.exp(-td / tau)
                else:
                    a = td + (2 * tau + td) * math.exp(-td / tau) - 2 * tau
                    ad = 1.0 - (1.0 + td / tau) * math.exp(-td / tau)
            else:
                e1, e2 = math.exp(-td / tau), math.exp(-(td - pw) / tau)
                if m == "lagstep1":
                    a, ad = pw + tau * e1 - tau * e2, -e1 + e2
                else:
                    a = pw + (2 * tau + td) * e1 + (pw - 2 * tau) * e2 - td * e2
                    ad = -(1.0 + td / tau) * e1 + (1.0 + (td - pw) / tau) * e2
            return (0.0, 0.0, a * ampr / pw, 0.0, 0.0, ad * ampr / pw)
        if m in ("eldredge", "eldredge1", "eldredge2"):
            # src/EldredgeManeuver.h:48-61 (pitch), src/Eldredge1.h:46-56 (plunge),
            # src/Eldredge2.h:52-71 (plunge velocity G, position its running integral)
            amp, a = p[0], p[1]
            q = (a,) + tuple(p[2:6])
            mx = _eld_max(a, a, *p[2:6])
            G, dG = _eld_G(*q, t), _eld_dG(*q, t)
            if m == "eldredge":
                r = amp * (pi / 180)
                return (0.0, 0.0, G * r / mx, 0.0, 0.0, dG * r / mx)
            if m == "eldredge1":
                return (0.0, G * amp / mx, 0.0, 0.0, dG * amp / mx, 0.0)
            h["g"] += G * (t - h["told"])
            h["told"] = t
            return (0.0, h["g"] * amp / mx, 0.0, 0.0, G * amp / mx, 0.0)
        if m == "eldredgecombined2":  # src/EldredgeCombined2.h:64-87
            ampa, a, a1, a2, a3, a4, ampb, b, b1, b2, b3, b4 = p
            mxa, mxb = _eld_max(a, a, a1, a2, a3, a4), _eld_max(b, a, b1, b2, b3, b4)
            Ga = _eld_G(a, a1, a2, a3, a4, t)
            h["g"] += Ga * (t - h["told"])
            h["told"] = t
            r = ampb * (pi / 180)
            return (0.0, h["g"] * ampa / mxa, _eld_G(b, b1, b2, b3, b4, t) * r / mxb, 0.0, Ga * ampa / mxa,
                    _eld_dG(b, b1, b2, b3, b4, t) * r / mxb)
        if m in ("motionfile", "motionfileperiodic"):  # src/MotionFile.h:90-115, src/MotionFilePeriodic.h:91-117
            tt = math.fmod(t, p[0]) if m == "motionfileperiodic" else t
            d = self.table
            idx = -1
            for i in range(len(d) - 1):  # the last interval holding tt, as the reference scans
                if d[i, 0] <= tt < d[i + 1, 0]:
                    idx = i
            if idx < 0:
                return (0.0,) * 6
            al = (tt - d[idx, 0]) / (d[idx + 1, 0] - d[idx, 0])
            return tuple(al * d[idx + 1, k] + (1 - al) * d[idx, k] for k in range(1, 7))
        return None

    def points_velocities(self, t: float):
        """RigidBody::moveBody: TangentSE2 mapPosition/mapVelocity about the centre."""
        tr = self.transformation(t)
        if tr is None:
            return self.ref_xy.copy(), np.zeros_like(self.ref_xy)
        x, y, th, xd, yd, thd = tr
        a = self.ref_xy[:, 0] - self.center[0]
        b = self.ref_xy[:, 1] - self.center[1]
        c, s = math.cos(th), math.sin(th)
        pos = np.stack([x + a * c - b * s + self.center[0], y + a * s + b * c + self.center[1]], axis=1)
        vel = np.stack([-a * s * thd - b * c * thd + xd, a * c * thd - b * s * thd + yd], axis=1)
        return pos, vel


def circle_points(xc, yc, r, n):
    """RigidBody::addCircle_n (src/RigidBody.cc:105-118)."""
    twopi = 8.0 * math.atan(1.0)
    dth = twopi / n
    i = np.arange(n)
    return np.stack([xc + r * np.cos(i * dth), yc + r * np.sin(i * dth)], axis=1)


def line_points(x1, y1, x2, y2, n):
    """RigidBody::addLine_n (src/RigidBody.cc:133-146)."""
    i = np.arange(n)
    dX = (x2 - x1) / (n - 1)
    dY = (y2 - y1) / (n - 1)
    return np.stack([x1 + i * dX, y1 + i * dY], axis=1)


# ----------------------------------------------------------------------------
# Model, projection, time stepping
# ----------------------------------------------------------------------------


SCHEMES = {  # (an, bn, cn) per sub-step (src/Scheme.h:13-61)
    "euler": [(1.0, 0.0, 1.0)],
    "ab2": [(3. / 2., -1. / 2., 1.0)],
    "rk3": [(8. / 15., 0.0, 8. / 15.), (5. / 12., -17. / 60., 2. / 3.), (3. / 4., -5. / 12., 1.0)],
    "rk3b": [(8. / 17., 0.0, 8. / 17.), (17. / 60., -15. / 68., 8. / 15.),
             (5. / 12., -17. / 60., 2. / 3.), (3. / 4., -5. / 12., 1.0)],
}


class Model:
    """NavierStokesModel (src/NavierStokesModel.cc:86-147) with the uniform base flow
    q0 = (U cos a dx_lev, U sin a dx_lev) (src/Flux.cc:79-99)."""

    def __init__(self, g: Grid, bodies: list, Re: float, u_mag: float = 1.0, alpha: float = 0.0):
        self.g, self.bodies, self.Re = g, bodies, Re
        self.poisson = EllipticSolver(g, "poisson")
        self.reg = Regularizer(g)
        self.q0 = g.flux()
        u, v = u_mag * math.cos(alpha), u_mag * math.sin(alpha)
        for lev in range(g.ngrid):
            dx = g.dx_lev(lev)
            self.q0[lev, : g.n_xflux] = u * dx
            self.q0[lev, g.n_xflux:] = v * dx
        self.npts = sum(b.ref_xy.shape[0] for b in bodies)
        self.time = 0.0
        self.u_mag, self.alpha_bf = u_mag, alpha
        self.frame = None      # the motion carried by the base flow (moving frame)
        self.move(0.0)

    @property
    def stationary(self) -> bool:
        return all(b.stationary for b in self.bodies)

    @property
    def time_dependent(self) -> bool:  # isTimeDependent (src/NavierStokesModel.cc:59-63)
        return not self.stationary or self.frame is not None

    def moving_frame(self) -> None:
        """The CLI's -ubf (src/ibpm.cc:166-178): Geometry::transferMotion (src/Geometry.cc:48-71) gives a
        fresh copy of the single moving body's motion to the base flow; the body keeps none."""
        if len(self.bodies) != 1:
            raise ValueError("the unsteady base flow needs exactly one body")
        b = self.bodies[0]
        if b.stationary:
            return
        self.frame = Body(b.ref_xy, b.center, b.motion, b.params, b.table)
        self.bodies[0] = Body(b.ref_xy, b.center)
        self.move(0.0)

    def move_flow(self, t: float) -> None:
        """BaseFlow::setAlphaMag + moveFlow (src/BaseFlow.cc:114-150) and Flux::setFlow (src/Flux.cc:101-129)."""
        x, y, th, xd, yd, thd = self.frame.transformation(t)
        xdT = xd - self.u_mag * math.cos(self.alpha_bf)
        ydT = yd - self.u_mag * math.sin(self.alpha_bf)
        gamma = math.atan2(ydT, -1.0 * xdT)
        alpha = -1.0 * th - gamma
        mag = math.sqrt(xdT * xdT + ydT * ydT)
        u, v, w = mag * math.cos(alpha), mag * math.sin(alpha), -1.0 * thd
        g = self.g
        xc, yc = self.frame.center
        for lev in range(g.ngrid):
            dx = g.dx_lev(lev)
            ycen = g.y_offset(lev) + (np.arange(g.ny) + 0.5) * dx     # x-flux y (getYCenter)
            xcen = g.x_offset(lev) + (np.arange(g.nx) + 0.5) * dx     # y-flux x (getXCenter)
            qx = np.broadcast_to((u - w * (ycen - yc)) * dx, (g.nx + 1, g.ny))
            qy = np.broadcast_to(((v + w * (xcen - xc)) * dx)[:, None], (g.nx, g.ny + 1))
            self.q0[lev, : g.n_xflux] = qx.reshape(-1)
            self.q0[lev, g.n_xflux:] = qy.reshape(-1)

    def move(self, t: float) -> None:
        pts, vel = [], []
        for b in self.bodies:
            p, v = b.points_velocities(t)
            pts.append(p)
            vel.append(v)
        self.points = np.concatenate(pts)
        self.velocities = np.concatenate(vel)
        self.reg.update(self.points)

    def update_operators(self, t: float) -> None:  # src/NavierStokesModel.cc:93-99
        if self.frame is not None:
            self.move_flow(t)
        if not self.stationary:
            self.move(t)

    @property
    def alpha(self) -> float:
        return 1.0 / self.Re

    def psi(self, w: np.ndarray) -> np.ndarray:
        """vorticityToStreamfunction: Poisson solve of -omega (src/NavierStokesModel.cc:133-140)."""
        return self.poisson.solve(coarsify(self.g, -1.0 * w))

    def flux_without_base(self, w):
        return curl_scalar(self.g, self.psi(w))

    def flux(self, w):  # computeFlux (src/NavierStokesModel.cc:121-125)
        return self.flux_without_base(w) + self.q0

    def B(self, f):  # src/NavierStokesModel.cc:101-105
        return curl_flux(self.g, self.reg.to_flux(f))

    def C(self, w):  # src/NavierStokesModel.cc:107-112
        return self.reg.to_boundary(self.flux_without_base(w))

    def constraints(self):  # getConstraints (src/NavierStokesModel.cc:86-91)
        b = np.concatenate([self.velocities[:, 0], self.velocities[:, 1]])
        return b - self.reg.to_boundary(self.q0)


class ProjectionSolver:
    """Fractional-step constrained solve (src/ProjectionSolver.cc:25-107) with a
    Cholesky (src/CholeskySolver.cc:49-224) or CG (src/ConjugateGradientSolver.cc:35-65)
    force solve."""

    def __init__(self, model: Model, beta: float, method: str = "cholesky", tol: float = 1e-7,
                 max_iter: int = 3000):
        self.model, self.beta, self.method = model, beta, method
        self.helm = EllipticSolver(model.g, "helmholtz", -beta / 2.0 * model.alpha)
        self.tol2 = tol * tol
        self.max_iter = max_iter
        self.last_iterations = 0
        self.L = None

    def Ainv(self, x):
        return self.helm.solve(x)

    def B(self, f):
        return self.model.B(f) * self.beta

    def C(self, x):
        return self.model.C(x)

    def M(self, f):
        return self.C(self.Ainv(self.B(f)))

    def matrix(self) -> np.ndarray:
        """Columns M e_j for all j at once (src/CholeskySolver.cc:63-79)."""
        m = 2 * self.model.npts
        E = np.eye(m)
        cols = self.M(E)          # (m, m): row j = M e_j
        return cols.T

    def init(self) -> None:
        if self.method != "cholesky":
            return
        M = self.matrix()
        # the reference reads the upper triangle M(i, j), j > i (src/CholeskySolver.cc:89-108)
        S = np.triu(M) + np.triu(M, 1).T
        self.L = np.linalg.cholesky(S)

    def Minv(self, b, x0):
        if self.method == "cholesky":
            import scipy.linalg as sla
            y = sla.solve_triangular(self.L, b, lower=True)
            return sla.solve_triangular(self.L.T, y, lower=False)
        # CG with warm start and absolute tolerance r.r <= tol^2
        x = x0.copy()
        r = b - self.M(x)
        d = r.copy()
        delta = float(r @ r)
        it = 0
        while delta > self.tol2 and it < self.max_iter:
            q = self.M(d)
            a = delta / float(d @ q)
            x = x + a * d
            r = r - a * q
            dold = delta
            delta = float(r @ r)
            d = r + (delta / dold) * d
            it += 1
        self.last_iterations = it
        return x

    def solve(self, a, b, f_prev):
        ws = self.Ainv(a)
        rhs = self.C(ws) - b
        f = self.Minv(rhs, f_prev)
        c = self.Ainv(self.B(f))
        return ws - c, f


@dataclass
class State:
    g: Grid
    npts: int
    omega: np.ndarray = None
    q: np.ndarray = None
    f: np.ndarray = None
    timestep: int = 0
    time: float = 0.0

    def __post_init__(self):
        if self.omega is None:
            self.omega = self.g.scalar()
        if self.q is None:
            self.q = self.g.flux()
        if self.f is None:
            self.f = np.zeros(2 * self.npts)

    def net_force(self):
        """State::computeNetForce (src/State.cc:53-63)."""
        n = self.npts
        dx2 = self.g.dx * self.g.dx
        return self.f[:n].sum() * dx2, self.f[n:].sum() * dx2


class IBSolver:
    """NonlinearIBSolver::advance / advanceSubstep (src/IBSolver.cc:142-198), and the other N(x)
    forms: `base` = list of (omega0, q0) for LinearizedIBSolver (one state) or
    LinearizedPeriodicIBSolver (one per phase); `sfd` = (chi, Delta, omega_hat) for SFDSolver
    (src/IBSolver.cc:238-283; omega_hat is the filtered vorticity it starts from)."""

    def __init__(self, model: Model, dt: float, scheme: str = "rk3", tol: float = 1e-7, max_iter: int = 3000,
                 base=None, sfd=None, adjoint=False):
        self.model, self.dt, self.coef = model, dt, SCHEMES[scheme]
        self.base = base
        self.adjoint = adjoint
        self.sfd = None
        if sfd is not None:
            chi, Delta, what = sfd
            self.sfd = dict(chi=chi, Delta=Delta, what=np.array(what, dtype=float), rhs_prev=None)
        method = "cholesky" if model.stationary else "cg"
        self.solvers = [ProjectionSolver(model, (an + bn) * dt, method, tol, max_iter)
                        for (an, bn, cn) in self.coef]
        self.Nprev = model.g.scalar()
        self.old_saved = False
        self.cg_iterations = []

    def init(self):
        for s in self.solvers:
            s.init()

    def advance(self, x: State) -> None:
        g, m = self.model.g, self.model
        for k, (an, bn, cn) in enumerate(self.coef):
            if self.base is not None:
                w0, q0 = self.base[x.timestep % len(self.base)]
                n = (adjoint if self.adjoint else linearized)(g, x.q, x.omega, q0, w0)
            else:
                n = nonlinear(g, x.q, x.omega)
            if self.sfd is not None:
                sf = self.sfd
                n = n - sf["chi"] * (x.omega - sf["what"])
                # the filtered state advances from the vorticity at the start of the sub-step
                rhs = (x.omega - sf["what"]) / sf["Delta"]
                a_f = an * rhs
                if bn != 0:
                    a_f = a_f + bn * (sf["rhs_prev"] if sf["rhs_prev"] is not None else rhs)
                sf["what"] = sf["what"] + a_f * self.dt
                sf["rhs_prev"] = rhs
            if m.time_dependent:
                m.update_operators(x.time + cn * self.dt)
            a = laplacian(g, x.omega) * (0.5 * m.alpha * (an + bn))
            a = a + an * n
            if bn != 0:
                if not self.old_saved:
                    self.Nprev = n
                a = a + bn * self.Nprev
            a = a * self.dt + x.omega
            b = m.constraints()
            x.omega, x.f = self.solvers[k].solve(a, b, x.f)
            self.cg_iterations.append(self.solvers[k].last_iterations)
            x.q = m.flux(x.omega)
            self.Nprev = n
            self.old_saved = True
        x.time += self.dt
        x.timestep += 1


# ----------------------------------------------------------------------------
# Inner products with multi-domain weights (src/VectorOperations.cc:222-412)
# ----------------------------------------------------------------------------


def scalar_ip_weights(g: Grid, fine_only: bool = False) -> np.ndarray:
    """Weight of every Scalar node in InnerProduct(Scalar, Scalar): dx^2 of its level,
    times 15/16 at the corners and 3/4 on the edges of the finer domain's footprint,
    0 inside it (src/VectorOperations.cc:222-310); FineGridInnerProduct keeps level 0."""
    nx, ny, nx2, ny2 = g.nx, g.ny, g.nxext, g.nyext
    w = np.zeros((g.ngrid, nx + 1, ny + 1))
    w[0, 1:nx, 1:ny] = 1.0
    if not fine_only:
        for lev in range(1, g.ngrid):
            W = w[lev]
            for (i, j) in ((nx2, ny2), (nx // 2 + nx2, ny2), (nx2, ny // 2 + ny2), (nx // 2 + nx2, ny // 2 + ny2)):
                W[i, j] += 15.0 / 16
            for j in range(ny2 + 1, ny // 2 + ny2):
                W[nx2, j] += 0.75
                W[nx // 2 + nx2, j] += 0.75
            for i in range(nx2 + 1, nx // 2 + nx2):
                W[i, ny2] += 0.75
                W[i, ny // 2 + ny2] += 0.75
            W[1:nx2, 1:ny] += 1.0
            W[nx // 2 + nx2 + 1:nx, 1:ny] += 1.0
            W[nx2:nx // 2 + nx2 + 1, 1:ny2] += 1.0
            W[nx2:nx // 2 + nx2 + 1, ny // 2 + ny2 + 1:ny] += 1.0
    for lev in range(g.ngrid):
        w[lev] *= (g.dx * 2 ** lev) ** 2
    return w[:, 1:nx, 1:ny]


def flux_ip_weights(g: Grid, fine_only: bool = False) -> np.ndarray:
    """Weight of every flux in InnerProduct(Flux, Flux) (src/VectorOperations.cc:312-412)."""
    nx, ny, nx2, ny2 = g.nx, g.ny, g.nxext, g.nyext
    nXf = (nx + 1) * ny
    w = np.zeros((g.ngrid, nXf + nx * (ny + 1)))
    X = lambda lev: w[lev, :nXf].reshape(nx + 1, ny)
    Y = lambda lev: w[lev, nXf:].reshape(nx, ny + 1)
    X(0)[1:nx, :] = 1.0
    Y(0)[:, 1:ny] = 1.0
    if not fine_only:
        for lev in range(1, g.ngrid):
            x, y = X(lev), Y(lev)
            x[nx2, ny2:ny // 2 + ny2] += 0.75
            x[nx // 2 + nx2, ny2:ny // 2 + ny2] += 0.75
            x[1:nx2, :] += 1.0
            x[nx // 2 + nx2 + 1:nx, :] += 1.0
            x[nx2:nx // 2 + nx2 + 1, 0:ny2] += 1.0
            x[nx2:nx // 2 + nx2 + 1, ny // 2 + ny2:ny] += 1.0
            y[nx2:nx // 2 + nx2, ny2] += 0.75
            y[nx2:nx // 2 + nx2, ny // 2 + ny2] += 0.75
            y[:, 1:ny2] += 1.0
            y[:, ny // 2 + ny2 + 1:ny] += 1.0
            y[0:nx2, ny2:ny // 2 + ny2 + 1] += 1.0
            y[nx // 2 + nx2:nx, ny2:ny // 2 + ny2 + 1] += 1.0
    return w


def inner_product(g: Grid, kind: int, a: np.ndarray, b: np.ndarray) -> float:
    """kind 0 InnerProduct(Scalar), 1 FineGridInnerProduct(Scalar), 2 InnerProduct(Flux),
    3 FineGridInnerProduct(Flux) (src/VectorOperations.cc:222-412)."""
    w = scalar_ip_weights(g, kind == 1) if kind < 2 else flux_ip_weights(g, kind == 3)
    return float(np.sum(w * np.asarray(a) * np.asarray(b)))


# ----------------------------------------------------------------------------
# Restart file (src/State.cc:65-223)
# ----------------------------------------------------------------------------


def save_restart(path: str, x: State, g: Grid) -> None:
    import struct
    with open(path, "wb") as fh:
        fh.write(struct.pack("iii", g.nx, g.ny, g.ngrid))
        fh.write(struct.pack("ddd", g.dx, g.x_offset(0), g.y_offset(0)))
        fh.write(struct.pack("i", x.npts))
        fh.write(np.ascontiguousarray(x.q, dtype="<f8").tobytes())
        fh.write(np.ascontiguousarray(x.omega, dtype="<f8").tobytes())
        n = x.npts
        fh.write(np.stack([x.f[:n], x.f[n:]], axis=1).astype("<f8").tobytes())
        fh.write(struct.pack("i", x.timestep))
        fh.write(struct.pack("d", x.time))


def load_restart(path: str):
    import struct
    with open(path, "rb") as fh:
        buf = fh.read()
    nx, ny, ngrid = struct.unpack_from("iii", buf, 0)
    dx, x0, y0 = struct.unpack_from("ddd", buf, 12)
    npts, = struct.unpack_from("i", buf, 36)
    off = 40
    F1 = 2 * nx * ny + nx + ny
    q = np.frombuffer(buf, "<f8", ngrid * F1, off).reshape(ngrid, F1).copy()
    off += 8 * ngrid * F1
    w = np.frombuffer(buf, "<f8", ngrid * (nx - 1) * (ny - 1), off).reshape(ngrid, nx - 1, ny - 1).copy()
    off += 8 * w.size
    fi = np.frombuffer(buf, "<f8", 2 * npts, off).reshape(npts, 2)
    off += 16 * npts
    f = np.concatenate([fi[:, 0], fi[:, 1]])
    timestep, = struct.unpack_from("i", buf, off)
    time, = struct.unpack_from("d", buf, off + 4)
    return dict(nx=nx, ny=ny, ngrid=ngrid, dx=dx, x0=x0, y0=y0, npts=npts, q=q, omega=w, f=f,
                timestep=timestep, time=time)
