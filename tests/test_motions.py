"""Rigid-body motions of the geometry file (src/RigidBody.cc:349-493).

CPU: the parser reads every `motion` keyword and motion files as the
reference does; the oracle's analytic motions have the derivatives they
claim and the piecewise ones are continuous.  The time-step parity of every
motion against fixtures the reference wrote runs with the other golden cases
(tests/test_gpu_parity.py, tests/test_oracle.py).

GPU: the device kinematics (positions and velocities of every boundary point)
against the oracle over a sequence of update times, including the history of
the stateful motions and motion-file ends; the learned preconditioner's
configuration sampling leaves that history untouched; the moving-frame base
flow (-ubf) refuses more than one body and ignores a fixed one.  Its
time-step parity runs with the golden cases (tests/golden/ubf_*.npz).
"""
import math

import numpy as np
import pytest

from helpers import FP64_TOL, golden_geometry, load_golden, oracle_from_golden, rel_l2
from ibpm_b200 import geometry as G
from oracle import ibpm_oracle as O

KINDS = ["fixedvel", "sigmoidalstep", "lagstep1", "lagstep2", "eldredge", "eldredge1", "eldredge2",
         "eldredgecombined2", "motionfile", "motionfileperiodic"]

PLATE = "body p\n  line 0 0 1 0 0.25\n  center 0.25 0\n  motion {}\nend\n"


def test_parser_reads_every_motion_keyword(tmp_path):
    (tmp_path / "m.txt").write_text("3\n0 0 0 0 1 2 3\n0.5 1 1 1 1 2 3\n1 2 2 2 1 2 3\n")
    lines = {"fixed 1 2 3": (G.MOTION_FIXED, 3), "fixedvel 1 2 3": (G.MOTION_FIXEDVEL, 3),
             "pitchplunge 1 2 3 4 5 6": (G.MOTION_PITCHPLUNGE, 6),
             "sigmoidalstep 1 2 3": (G.MOTION_SIGMOIDALSTEP, 3), "LagStep1 1 2 3 4": (G.MOTION_LAGSTEP1, 4),
             "lagstep2 1 2 3 4": (G.MOTION_LAGSTEP2, 4), "eldredge 1 2 3 4 5 6": (G.MOTION_ELDREDGE, 6),
             "eldredgecombined2 " + " ".join(str(k) for k in range(1, 13)): (G.MOTION_ELDREDGECOMBINED2, 12),
             "eldredge1 1 2 3 4 5 6": (G.MOTION_ELDREDGE1, 6), "eldredge2 1 2 3 4 5 6": (G.MOTION_ELDREDGE2, 6),
             "motionfile m.txt": (G.MOTION_FILE, 0), "motionfileperiodic m.txt 0.75": (G.MOTION_FILE_PERIODIC, 1)}
    for line, (code, npar) in lines.items():
        b = G.parse(PLATE.format(line), str(tmp_path)).bodies[0]
        assert b.motion == code and len(b.params) == npar, line
        assert b.stationary == (code == G.MOTION_FIXED)
        assert len(b.points) == 5 and b.center == (0.25, 0.0)
        if code in (G.MOTION_FILE, G.MOTION_FILE_PERIODIC):
            assert b.table.shape == (3, 7) and b.table[2, 1] == 2.0
    assert G.parse(PLATE.format("motionfileperiodic m.txt 0.75"), str(tmp_path)).bodies[0].params == (0.75,)


def test_parser_rejects_bad_motions(tmp_path):
    (tmp_path / "bad.txt").write_text("2\n0 0 0 0 0 0 0\n")
    (tmp_path / "back.txt").write_text("2\n1 0 0 0 0 0 0\n0.5 0 0 0 0 0 0\n")
    for line in ("pitchplunge 1 2 3", "unknownmotion 1", "eldredge 1 2 3 4 5", "motionfile bad.txt",
                 "motionfile back.txt", "motionfile missing.txt", "fixedvel a b c"):
        with pytest.raises((G.GeometryError, OSError)):
            G.parse(PLATE.format(line), str(tmp_path))


def _body(kind, params, table=None):
    return O.Body(np.array([[0.0, 0.0], [1.0, 0.0]]), (0.25, 0.0), kind, tuple(params), table)


def _fd_check(kind, params, times, comps=(0, 1, 2)):
    """d/dt of (x, y, theta) against the velocities the motion returns."""
    h = 1e-7
    for t in times:
        tr = _body(kind, params).transformation(t)
        p = _body(kind, params).transformation(t + h)
        m = _body(kind, params).transformation(t - h)
        for k in comps:
            fd = (p[k] - m[k]) / (2 * h)
            assert abs(fd - tr[3 + k]) <= 1e-5 * max(1.0, abs(fd)), (kind, t, k, fd, tr[3 + k])


def test_oracle_analytic_motions_are_consistent():
    ts = [-0.01, 0.004, 0.013, 0.021, 0.034, 0.049, 0.08]
    _fd_check("sigmoidalstep", (15, 0.08, 0.005), ts)
    _fd_check("lagstep1", (5, 0.03, 0.01, 0.005), [t for t in ts if abs(t - 0.005) > 1e-6 and abs(t - 0.035) > 1e-6])
    _fd_check("lagstep2", (5, 0.03, 0.008, 0.004), [t for t in ts if abs(t - 0.004) > 1e-6])
    _fd_check("eldredge", (10, 120, 0.005, 0.02, 0.035, 0.05), ts)
    _fd_check("eldredge1", (0.05, 120, 0.005, 0.02, 0.035, 0.05), ts)
    _fd_check("pitchplunge", (0.3, 0.5, 0.1, 0.2, 0.4, 0.0), ts)
    # the lag steps are continuous at the pulse end, and reach the ramp's plateau
    for kind, p in (("lagstep1", (5, 0.03, 0.01, 0.0)), ("lagstep2", (5, 0.03, 0.008, 0.0))):
        a = _body(kind, p).transformation(0.03 - 1e-12)
        b = _body(kind, p).transformation(0.03 + 1e-12)
        assert abs(a[2] - b[2]) < 1e-9 and abs(a[5] - b[5]) < 1e-6
        assert abs(_body(kind, p).transformation(5.0)[2] - math.radians(5)) < 1e-12
    # Eldredge's ramp is normalised to its amplitude at mid-plateau
    tr = _body("eldredge", (10, 120, 0.005, 0.02, 0.035, 0.05)).transformation(0.0275)
    assert abs(tr[2] - math.radians(10)) < 1e-12


def test_oracle_stateful_motions_follow_the_call_history():
    # FixedVelocity integrates over the calls and drops steps longer than one time unit
    b = _body("fixedvel", (0.4, -0.25, 0.8))
    for t in (0.0, 0.3, 0.3, 0.9, 2.5, 2.7):
        tr = b.transformation(t)
    assert np.allclose(tr[:3], (0.4 * 1.1, -0.25 * 1.1, 0.8 * 1.1)) and tr[3:] == (0.4, -0.25, 0.8)
    # Eldredge2's position is the right-endpoint sum of its velocity over the calls
    p = (0.5, 120, 0.005, 0.02, 0.035, 0.05)
    b = _body("eldredge2", p)
    ts = np.linspace(0.0, 0.06, 25)
    ys = [b.transformation(t)[1] for t in ts]
    mx = O._eld_max(120, 120, 0.005, 0.02, 0.035, 0.05)
    vel = np.array([O._eld_G(120, 0.005, 0.02, 0.035, 0.05, t) * 0.5 / mx for t in ts])
    assert abs(ys[-1] - np.sum(vel[1:] * np.diff(ts))) < 1e-12


def test_oracle_motion_file_interpolates_and_wraps():
    tab = np.array([[0.0, 0, 0, 0, 0, 0, 0], [0.5, 1, 2, 3, 4, 5, 6], [1.0, 3, 2, 1, 0, 0, 0]])
    b = _body("motionfile", (), tab)
    assert np.allclose(b.transformation(0.25), (0.5, 1, 1.5, 2, 2.5, 3))
    assert np.allclose(b.transformation(0.75), (2, 2, 2, 2, 2.5, 3))
    assert b.transformation(1.0) == (0.0,) * 6 and b.transformation(-0.1) == (0.0,) * 6
    bp = _body("motionfileperiodic", (0.6,), tab)
    assert np.allclose(bp.transformation(0.85), b.transformation(0.25))


# --------------------------------------------------------------------------- GPU


def _device_and_oracle(kind, **kw):
    import ibpm_b200 as ib
    d = load_golden("motion_" + kind)
    grid = ib.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
                   float(d["yoffset"]))
    geo = golden_geometry(d)
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, float(d["Re"])), float(d["dt"]), "rk3",
                             float(d["tol"]), **kw)
    return ib, d, grid, geo, s


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
def test_device_kinematics_match_oracle(kind):
    ib, d, grid, geo, s = _device_and_oracle(kind)
    g, model, solver, x = oracle_from_golden(d)   # both moved to t = 0 on construction
    # (cosh(a t) of the Eldredge ramps overflows near a t = 710, in the reference too: a = 120 stops at t = 2.6)
    for t in (0.0, 0.0037, 0.011, 0.011, 0.0213, 0.029, 0.047, 0.068, 0.5, 2.25, 2.6):
        s.update_operators(t)
        model.update_operators(t)
        pts, vel = s.boundary()
        assert np.max(np.abs(pts - model.points)) < 1e-12, (kind, t)
        assert np.max(np.abs(vel - model.velocities)) < 1e-10 * max(1.0, np.max(np.abs(model.velocities))), (kind, t)
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["eldredge2", "fixedvel"])
def test_configuration_sampling_keeps_motion_history(kind):
    """Sampling body configurations for the learned preconditioner moves the
    bodies to other times; the stateful motions' history must not see it."""
    ib, d, grid, geo, s = _device_and_oracle(kind)
    s.lpc_generate(3, 0.013, 0.041)
    x = ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float))
    s.init()
    s.set_state(x, with_q=False)
    n = int(d["nsteps"])
    s.advance_resident(n)
    assert rel_l2(s.force_history(n), d["forces"][:, 2:4]) < FP64_TOL
    s.get_state(x)
    assert rel_l2(x.omega, d["omega"]) < FP64_TOL
    s.close()


def test_oracle_moving_frame_flow_is_the_relative_free_stream():
    """-ubf with a translating body: the base flow is the free stream minus the body's velocity, in the
    body's frame; the body itself stays at its reference points."""
    g = O.Grid(32, 16, 2, 4.0, -2.0, -1.0)
    b = O.Body(np.array([[0.0, 0.0], [0.5, 0.0]]), (0.0, 0.0), "fixedvel", (0.4, -0.25, 0.0))
    m = O.Model(g, [b], 100.0)
    m.moving_frame()
    assert m.stationary and m.time_dependent
    m.update_operators(0.3)
    for lev in range(g.ngrid):
        dx = g.dx_lev(lev)
        assert np.allclose(m.q0[lev, : g.n_xflux], 0.6 * dx, rtol=0, atol=1e-15)
        assert np.allclose(m.q0[lev, g.n_xflux:], 0.25 * dx, rtol=0, atol=1e-15)
    assert np.array_equal(m.points, b.ref_xy)
    with pytest.raises(ValueError):
        O.Model(g, [b, O.Body(np.array([[1.0, 0.5]]))], 100.0).moving_frame()


@pytest.mark.gpu
def test_moving_frame_needs_one_body_and_ignores_a_fixed_one():
    """ibg_set_moving_frame refuses two bodies, as the reference CLI exits; a fixed body keeps the
    steady base flow (the reference ignores the flag) and the run stays the reference's."""
    import ibpm_b200 as ib
    d = load_golden("cyl_l1_rk3")
    grid = ib.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
                   float(d["yoffset"]))
    geo = golden_geometry(d)
    two = G.Geometry(geo.bodies + [G.RigidBody(points=[(1.5, 1.5)], motion=G.MOTION_FIXEDVEL,
                                               params=(0.1, 0.0, 0.0))])
    with pytest.raises(ib.IbgError):
        ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, two, float(d["Re"]), ubf=True), float(d["dt"]))
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, float(d["Re"]), ubf=True), float(d["dt"]),
                             str(d["scheme"]), float(d["tol"]))
    x = ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float))
    s.init()
    s.set_state(x, with_q=False)
    n = int(d["nsteps"])
    s.advance_resident(n)
    assert rel_l2(s.force_history(n), d["forces"][:, 2:4]) < FP64_TOL
    s.close()


@pytest.mark.gpu
def test_create_rejects_degenerate_motions():
    """ibg_create refuses motions whose reference formulas would divide by zero or that are not
    well formed (the reference would step on with infinities): a zero sigmoid duration, a zero lag
    time constant, an Eldredge ramp with no plateau, a motion file running backwards in time."""
    import ibpm_b200 as ib
    grid = ib.Grid(32, 32, 1, 4.0, -2.0, -2.0)
    pts = [(x, 0.0) for x in np.linspace(-0.5, 0.5, 9)]
    bad = [(G.MOTION_SIGMOIDALSTEP, (15.0, 0.0, 0.0), None),
           (G.MOTION_LAGSTEP1, (5.0, 0.03, 0.0, 0.0), None),
           (G.MOTION_ELDREDGE, (10.0, 50.0, 0.1, 0.1, 0.1, 0.1), None),
           (G.MOTION_FILE, (), np.array([[0.1, 0, 0, 0, 0, 0, 0], [0.0, 0, 0, 0, 0, 0, 0]])),
           (G.MOTION_PITCHPLUNGE, (float("nan"), 0.5, 0.0, 0.1, 0.5, 0.0), None)]
    for code, params, table in bad:
        body = G.RigidBody(points=list(pts), center=(0.0, 0.0), motion=code, params=params, table=table)
        model = ib.NavierStokesModel(grid, G.Geometry([body]), 100.0)
        with pytest.raises(ib.IbgError):
            ib.NonlinearIBSolver(grid, model, 0.01)
    # an empty motion file is the reference's zero transformation: the body stays where it is
    body = G.RigidBody(points=list(pts), center=(0.0, 0.0), motion=G.MOTION_FILE, params=(),
                       table=np.zeros((0, 7)))
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, G.Geometry([body]), 100.0), 0.01)
    s.update_operators(0.37)
    p, v = s.boundary()
    assert np.array_equal(p, np.array(pts)) and not np.any(v)
    s.close()


def test_oracle_moving_frame_flow_is_divergence_free_rigid_motion():
    """A rotating frame's base flow is rigid: on every level the discrete divergence of q0 vanishes
    and its vorticity is the same at every interior node, -2 thetadot (seen from the body, the flow
    turns the other way)."""
    g = O.Grid(32, 16, 2, 4.0, -2.0, -1.0)
    b = O.Body(np.array([[0.0, 0.0], [0.5, 0.0]]), (0.1, -0.05), "fixedvel", (0.3, 0.1, 0.7))
    m = O.Model(g, [b], 100.0)
    m.moving_frame()
    m.update_operators(0.2)
    for lev in range(g.ngrid):
        qx = m.q0[lev, : g.n_xflux].reshape(g.nx + 1, g.ny)
        qy = m.q0[lev, g.n_xflux:].reshape(g.nx, g.ny + 1)
        div = (qx[1:, :] - qx[:-1, :]) + (qy[:, 1:] - qy[:, :-1])
        assert np.max(np.abs(div)) < 1e-14
        # circulation around each interior node's dual cell, per unit area: the same everywhere
        dx = g.dx_lev(lev)
        circ = (qy[1:, 1:-1] - qy[:-1, 1:-1]) - (qx[1:-1, 1:] - qx[1:-1, :-1])
        assert np.ptp(circ) < 1e-13 and abs(circ.mean() / (dx * dx) + 2 * 0.7) < 1e-12
