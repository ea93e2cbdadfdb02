"""Parity of the CUDA time step (through the C ABI) with the oracle.

The oracle is the numpy restatement in oracle/ibpm_oracle.py, itself pinned
to the reference library; the golden fixtures in tests/golden/ come from the
reference library directly.  FP64 bar: relative L2 <= 1e-10 (operators
<= 1e-12).
"""
import numpy as np
import pytest

from helpers import FP64_TOL, golden_geometry, golden_names, load_golden, oracle_from_golden, rel_l2

pytestmark = pytest.mark.gpu

OP_TOL = 1e-12


def _solver_for(gp, pts, Re=100.0, dt=0.01, scheme="rk3", motion=None, tol=1e-7):
    import ibpm_b200 as ib
    from ibpm_b200 import geometry
    grid = ib.Grid(*gp)
    body = geometry.RigidBody(points=[tuple(p) for p in pts])
    if motion is not None:
        body.motion, body.params, body.center = motion
    geo = geometry.Geometry([body])
    model = ib.NavierStokesModel(grid, geo, Re)
    return grid, model, ib.NonlinearIBSolver(grid, model, dt, scheme, tol)


# (the odd single-level grids give odd lengths N = nx, ny to the FP64 half-length DSTs, whose last sine
# sum then has no even partner)
GRIDS = [(16, 16, 1, 2.0, -1.0, -1.0), (32, 16, 3, 3.0, -1.5, -0.75), (64, 64, 2, 4.0, -2.0, -2.0),
         (40, 24, 4, 2.0, -1.0, -0.6), (45, 27, 1, 3.0, -1.5, -0.9), (21, 35, 1, 2.0, -1.0, -1.6)]


@pytest.mark.parametrize("gp", GRIDS)
def test_elliptic_and_stencils(gp):
    from oracle import ibpm_oracle as O
    g = O.Grid(*gp)
    pts = O.circle_points(0.0, 0.0, 0.2 * gp[3] / 2, 12)
    grid, model, s = _solver_for(gp, pts)
    rng = np.random.default_rng(sum(gp[:3]))
    f = rng.standard_normal(g.scalar().shape)
    q = rng.standard_normal(g.flux().shape)
    assert rel_l2(s.poisson(f), O.EllipticSolver(g, "poisson").solve(f)) < OP_TOL
    assert rel_l2(s.helmholtz(-0.0123, f), O.EllipticSolver(g, "helmholtz", -0.0123).solve(f)) < OP_TOL
    assert rel_l2(s.nonlinear(q, f), O.nonlinear(g, q, f)) < OP_TOL
    assert rel_l2(s.laplacian(f), O.laplacian(g, f)) < OP_TOL
    reg = O.Regularizer(g)
    reg.update(pts)
    fb = rng.standard_normal(2 * len(pts))
    assert rel_l2(s.model_B(fb), O.curl_flux(g, reg.to_flux(fb))) < OP_TOL
    model_o = O.Model(g, [O.Body(pts)], 100.0)
    assert rel_l2(s.model_C(f), model_o.C(f)) < OP_TOL
    assert rel_l2(s.reg_to_boundary(q[0]), reg.to_boundary(q)) < OP_TOL
    assert rel_l2(s.reg_to_flux(fb), reg.to_flux(fb)) < OP_TOL
    s.close()


# grids whose DST lengths 2 nx and 2 ny have compile-time FFT plans (256, 384, 400, 512, 768, 800, 1000,
# 1024, 2048; the small grids above take the general path)
COMPILED_FFT_GRIDS = [(128, 192, 2, 4.0, -2.0, -3.0), (256, 200, 3, 4.0, -2.0, -1.5625),
                      (500, 200, 2, 10.0, -5.0, -2.0), (384, 512, 2, 6.0, -3.0, -4.0), (1024, 128, 2, 8.0, -4.0, -0.5)]


@pytest.mark.parametrize("gp", GRIDS + COMPILED_FFT_GRIDS[:2])
@pytest.mark.parametrize("half", [0, 1])
def test_both_fp64_dst_forms_match_oracle(gp, half):
    """The FP64 passes and sweep lines in either DST form (half-length FFTs or the odd extension; a
    context picks one per grid by timing) against the oracle's multi-domain solves."""
    from oracle import ibpm_oracle as O
    from ibpm_b200 import _native
    g = O.Grid(*gp)
    grid, model, s = _solver_for(gp, O.circle_points(0.0, 0.0, 0.2 * gp[3] / 2, 12))
    assert _native.lib().ibg_set_pass_form(s.handle, half) == 0
    rng = np.random.default_rng(gp[0] + 3 * gp[1] + half)
    f = rng.standard_normal(g.scalar().shape)
    assert rel_l2(s.poisson(f), O.EllipticSolver(g, "poisson").solve(f)) < OP_TOL
    assert rel_l2(s.helmholtz(-0.0123, f), O.EllipticSolver(g, "helmholtz", -0.0123).solve(f)) < OP_TOL
    s.close()


@pytest.mark.parametrize("gp", COMPILED_FFT_GRIDS)
def test_compiled_fft_lengths_match_oracle(gp):
    from oracle import ibpm_oracle as O
    g = O.Grid(*gp)
    grid, model, s = _solver_for(gp, O.circle_points(0.0, 0.0, 0.3, 24))
    rng = np.random.default_rng(gp[0] + gp[1])
    f = rng.standard_normal(g.scalar().shape)
    assert rel_l2(s.poisson(f), O.EllipticSolver(g, "poisson").solve(f)) < OP_TOL
    assert rel_l2(s.helmholtz(-0.0123, f), O.EllipticSolver(g, "helmholtz", -0.0123).solve(f)) < OP_TOL
    s.close()


def test_multidomain_inverse_property_full_size():
    """L(solve(f)) = coarsify(f) on every level at the 400x200, 5-level size
    (the reference's EllipticSolverTest property, src test/EllipticSolverTest.cc:86-121)."""
    from oracle import ibpm_oracle as O
    gp = (400, 200, 5, 8.0, -2.0, -2.0)
    g = O.Grid(*gp)
    grid, model, s = _solver_for(gp, O.circle_points(0, 0, 0.5, 157))
    rng = np.random.default_rng(0)
    f = rng.standard_normal(g.scalar().shape)
    u = s.poisson(f)
    Lu = s.laplacian(u)
    cf = O.coarsify(g, f)
    # the multi-domain Laplacian uses boundary values from the coarser level, exactly as the solve
    assert rel_l2(Lu, cf) < 1e-9
    s.close()


def test_projection_matches_oracle():
    from oracle import ibpm_oracle as O
    gp = (48, 32, 2, 3.0, -1.5, -1.0)
    g = O.Grid(*gp)
    pts = O.circle_points(0.1, 0.05, 0.35, 24)
    grid, model, s = _solver_for(gp, pts, Re=150.0, dt=0.02)
    s.init()
    mo = O.Model(g, [O.Body(pts)], 150.0)
    rng = np.random.default_rng(5)
    a = rng.standard_normal(g.scalar().shape)
    b = rng.standard_normal(48)
    beta0 = (8. / 15.) * 0.02
    ps = O.ProjectionSolver(mo, beta0)
    ps.init()
    w_o, f_o = ps.solve(a, b, np.zeros(48))
    w_g, f_g = s.projection_solve(0, a, b, np.zeros(48))
    assert rel_l2(w_g, w_o) < 1e-11
    assert rel_l2(f_g, f_o) < 1e-10
    s.close()


@pytest.mark.parametrize("name", golden_names())
def test_time_step_matches_reference_golden(name):
    import ibpm_b200 as ib
    d = load_golden(name)
    grid = ib.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
                   float(d["yoffset"]))
    geo = golden_geometry(d)
    model = ib.NavierStokesModel(grid, geo, float(d["Re"]), ubf=bool(int(d.get("ubf", 0))))
    s = ib.NonlinearIBSolver(grid, model, float(d["dt"]), str(d["scheme"]), float(d["tol"]))
    x = ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float))
    s.init()
    s.set_state(x, with_q=False)
    n = int(d["nsteps"])
    s.advance_resident(n)
    forces = s.force_history(n)
    s.get_state(x)
    assert rel_l2(forces, d["forces"][:, 2:4]) < FP64_TOL
    assert rel_l2(x.omega, d["omega"]) < FP64_TOL
    assert rel_l2(x.q, d["q"]) < FP64_TOL
    assert rel_l2(x.f, d["f"]) < 1e-9
    assert x.timestep == int(d["timestep"])
    assert abs(x.time - float(d["time"])) < 1e-12
    s.close()


def test_drop_in_advance_keeps_host_state():
    """advance(State&) leaves the host State valid after every call, like the reference."""
    import ibpm_b200 as ib
    d = load_golden("cyl_l1_rk3")
    grid = ib.Grid(48, 48, 1, 4.0, -2.0, -2.0)
    geo = ib.geometry.parse(str(d["geom"]))
    model = ib.NavierStokesModel(grid, geo, float(d["Re"]))
    s = ib.NonlinearIBSolver(grid, model, float(d["dt"]), "rk3")
    s.init()
    x = ib.State(grid, geo.num_points)
    s.refresh_state(x)
    F = []
    for _ in range(int(d["nsteps"])):
        s.advance(x)
        F.append(x.computeNetForce())
    assert rel_l2(np.array(F), d["forces"][:, 2:4]) < FP64_TOL
    assert rel_l2(x.omega, d["omega"]) < FP64_TOL
    s.close()


def test_cholesky_save_load_roundtrip(tmp_path):
    import ibpm_b200 as ib
    d = load_golden("cyl_l1_rk3")
    grid = ib.Grid(48, 48, 1, 4.0, -2.0, -2.0)
    geo = ib.geometry.parse(str(d["geom"]))
    model = ib.NavierStokesModel(grid, geo, float(d["Re"]))
    s = ib.NonlinearIBSolver(grid, model, float(d["dt"]), "rk3")
    s.init()
    base = str(tmp_path / "run")
    assert s.save(base)
    s2 = ib.NonlinearIBSolver(grid, model, float(d["dt"]), "rk3")
    assert s2.load(base)
    x = ib.State(grid, geo.num_points)
    s2.set_state(x, with_q=False)
    s2.advance_resident(int(d["nsteps"]))
    assert rel_l2(s2.force_history(int(d["nsteps"])), d["forces"][:, 2:4]) < FP64_TOL
    # a factor for another dt is rejected (src/CholeskySolver.cc:131-136)
    s3 = ib.NonlinearIBSolver(grid, model, float(d["dt"]) * 2, "rk3")
    assert not s3.load(base)
    for h in (s, s2, s3):
        h.close()


def test_c1_size_steps_match_oracle():
    """The 200x200 fixed-cylinder workload: a few steps against the oracle."""
    from ibpm_b200 import configs
    import ibpm_b200 as ib
    from oracle import ibpm_oracle as O
    wl = configs.c1_fixed_cylinder()
    grid, model, s, x = ib.from_workload(wl)
    s.init()
    s.set_state(x, with_q=False)
    nsteps = 4
    s.advance_resident(nsteps)
    fg = s.force_history(nsteps)
    s.get_state(x)
    g = O.Grid(wl.nx, wl.ny, wl.ngrid, wl.length, wl.xoffset, wl.yoffset)
    geo = ib.geometry.parse(wl.geom)
    mo = O.Model(g, [O.Body(np.array(geo.bodies[0].points))], wl.Re)
    so = O.IBSolver(mo, wl.dt, "rk3")
    so.init()
    xo = O.State(g, mo.npts)
    xo.q = mo.flux(xo.omega)
    fo = []
    for _ in range(nsteps):
        so.advance(xo)
        fo.append(xo.net_force())
    assert rel_l2(fg, np.array(fo)) < FP64_TOL
    assert rel_l2(x.omega, xo.omega) < FP64_TOL
    s.close()


@pytest.mark.parametrize("precision", ["fp32_refined", "fp32"])
@pytest.mark.parametrize("name", ["cyl_l3_noise_rk3", "plate_l2_pitchplunge_cg"])
def test_reduced_precision_forms_against_reference(name, precision):
    """The reduced-precision forms against the reference run.  fp32_refined
    (FP32 transforms with one FP64-residual refinement per solve, FP64 state)
    is held to the bars of the reduced-precision form: vorticity within 1e-5
    and forces within 1e-4 relative.  fp32 (the whole bulk in FP32, no
    refinement) keeps vorticity within 1e-5 but its forces only within 3e-4 on
    these short runs from rest: the constraint right-hand side C w* - b is a
    small difference of O(1) terms and M^-1 amplifies the FP32 state error."""
    import ibpm_b200 as ib
    d = load_golden(name)
    grid = ib.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
                   float(d["yoffset"]))
    geo = ib.geometry.parse(str(d["geom"]))
    model = ib.NavierStokesModel(grid, geo, float(d["Re"]))
    s = ib.NonlinearIBSolver(grid, model, float(d["dt"]), str(d["scheme"]), max(float(d["tol"]), 1e-7),
                             precision=precision)
    x = ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float))
    s.init()
    s.set_state(x, with_q=False)
    n = int(d["nsteps"])
    s.advance_resident(n)
    forces = s.force_history(n)
    s.get_state(x)
    assert rel_l2(forces, d["forces"][:, 2:4]) < (1e-4 if precision == "fp32_refined" else 3e-4)
    assert rel_l2(x.omega, d["omega"]) < 1e-5
    s.close()


@pytest.mark.parametrize("member", [13, 29])
def test_fp32_member_forces_within_1e4(member):
    """An FP32-bulk ensemble member (a 512x512 single-domain and a 128x128 two-domain ellipse) against
    the same member in FP64: forces within 1e-4 over 12 steps from rest.  In float, the eigenvalues'
    cos + cos - 2 cancels for the low modes; the FP32 tables hold cos - 1 instead."""
    import ibpm_b200 as ib
    from ibpm_b200 import configs
    wl = configs.ensemble_members(count=64)[member]
    n = 12
    F = {}
    for prec in ("fp64", "fp32"):
        grid, model, s, x = ib.from_workload(wl, precision=prec)
        s.init()
        s.set_state(x, with_q=False)
        s.advance_resident(n)
        F[prec] = s.force_history(n)
        s.close()
    assert rel_l2(F["fp32"], F["fp64"]) < 1e-4


def test_ensemble_matches_members_stepped_alone():
    """Members advanced by one ensemble graph give the same forces and
    vorticity as the same members advanced one by one."""
    import ibpm_b200 as ib
    from ibpm_b200 import configs
    specs = [(32, 32, 2, 3.0, -1.5, -1.5, 24, 0.4, 150.0, 0.02), (48, 48, 1, 4.0, -2.0, -2.0, 36, 0.5, 100.0, 0.02),
             (64, 32, 3, 4.0, -1.5, -1.0, 32, 0.4, 200.0, 0.01)]

    def make():
        out = []
        for (nx, ny, L, length, xo, yo, npts, r, Re, dt) in specs:
            grid = ib.Grid(nx, ny, L, length, xo, yo)
            geo = ib.geometry.parse(configs.cylinder_geom(npts, r=r))
            s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, Re), dt, "rk3")
            s.init()
            s.set_state(ib.State(grid, geo.num_points), with_q=False)
            out.append((s, grid, geo))
        return out

    nsteps = 5
    alone = make()
    for s, _, _ in alone:
        s.advance_resident(nsteps)
    together = make()
    ens = ib.Ensemble([s for s, _, _ in together])
    ens.advance(nsteps)
    for (sa, grid, geo), (sb, _, _) in zip(alone, together):
        fa, fb = sa.force_history(nsteps), sb.force_history(nsteps)
        assert rel_l2(fb, fa) < 1e-12
        xa, xb = ib.State(grid, geo.num_points), ib.State(grid, geo.num_points)
        sa.get_state(xa)
        sb.get_state(xb)
        assert rel_l2(xb.omega, xa.omega) < 1e-12
    ens.close()
    for s, _, _ in alone + together:
        s.close()


@pytest.mark.parametrize("name", ["plate_l2_pitchplunge_cg", "plate_l3_ny2mod4_cg"])
def test_cholesky_preconditioned_cg_matches_reference(name):
    """PCG with the refreshed-Cholesky preconditioner converges to the same
    absolute tolerance as the reference's CG in fewer iterations."""
    import ibpm_b200 as ib
    d = load_golden(name)
    grid = ib.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
                   float(d["yoffset"]))
    geo = ib.geometry.parse(str(d["geom"]))
    model = ib.NavierStokesModel(grid, geo, float(d["Re"]))
    its = {}
    for pc in ("none", "cholesky"):
        s = ib.NonlinearIBSolver(grid, model, float(d["dt"]), str(d["scheme"]), float(d["tol"]), precond=pc,
                                 pc_refresh=2)
        x = ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float))
        s.init()
        s.set_state(x, with_q=False)
        n = int(d["nsteps"])
        s.advance_resident(n)
        forces = s.force_history(n)
        s.get_state(x)
        its[pc] = s.cg_totals()[0]
        assert rel_l2(forces, d["forces"][:, 2:4]) < 1e-8
        assert rel_l2(x.omega, d["omega"]) < 1e-9
        s.close()
    assert its["cholesky"] * 3 < its["none"], its


def test_host_driven_cg_loop_matches_reference():
    """The host-driven CG loop (no device-side WHILE node) on the moving plate."""
    import ibpm_b200 as ib
    d = load_golden("plate_l2_pitchplunge_cg")
    grid = ib.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
                   float(d["yoffset"]))
    geo = ib.geometry.parse(str(d["geom"]))
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, float(d["Re"])), float(d["dt"]), "rk3",
                             float(d["tol"]), cg_graph=False)
    x = ib.State(grid, geo.num_points)
    s.init()
    s.set_state(x, with_q=False)
    n = int(d["nsteps"])
    s.advance_resident(n)
    assert rel_l2(s.force_history(n), d["forces"][:, 2:4]) < FP64_TOL
    s.close()


def test_contexts_of_different_sizes_coexist():
    """Kernel shared-memory limits are per process: a context created after
    another with a smaller grid must not break the larger one's launches."""
    import ibpm_b200 as ib
    from ibpm_b200 import configs

    def make(n, L):
        grid = ib.Grid(n, n, L, 4.0, -2.0, -2.0)
        geo = ib.geometry.parse(configs.cylinder_geom(48, r=0.4))
        s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, 100.0), 0.005, "rk3")
        s.init()
        s.set_state(ib.State(grid, geo.num_points), with_q=False)
        return s

    alone = make(384, 2)
    alone.advance_resident(3)
    fa = alone.force_history(3)
    alone.close()
    big = make(384, 2)
    small = make(64, 1)
    big.advance_resident(3)
    small.advance_resident(3)
    assert rel_l2(big.force_history(3), fa) < 1e-13
    big.close()
    small.close()


def test_autotuner_records_valid_shapes():
    """Creating a context times the DST passes' launch shapes once per grid shape."""
    import ibpm_b200 as ib
    from ibpm_b200 import configs
    grid = ib.Grid(96, 64, 2, 4.0, -2.0, -2.0)
    geo = ib.geometry.parse(configs.cylinder_geom(40, r=0.4))
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, 100.0), 0.01, "rk3")
    log = ib.autotune_log()
    mine = [r for r in log if r["levels"] == 2 and r["lines"] in (95, 63) and r["bytes"] == 8]
    assert {r["pass"] for r in mine} == {0, 1}
    for r in mine:
        assert r["pairs_per_cta"] in (1, 2, 4) and r["threads"] in (128, 256, 512)
        assert r["twiddles_in_smem"] in (0, 1)
    s.close()


def test_ensemble_shapes_do_not_change_results():
    """Setting one launch shape for every member recaptures the members' steps; the
    results stay those of the members run alone."""
    import ibpm_b200 as ib
    from ibpm_b200 import configs

    def make():
        grid = ib.Grid(64, 64, 2, 4.0, -2.0, -2.0)
        geo = ib.geometry.parse(configs.cylinder_geom(48, r=0.4))
        s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, 150.0), 0.01, "rk3")
        s.init()
        s.set_state(ib.State(grid, geo.num_points), with_q=False)
        return s

    alone = make()
    alone.advance_resident(8)
    fa = alone.force_history(8)
    a, b = make(), make()
    ens = ib.Ensemble([a, b])
    ens.advance(2)
    ens.set_shapes(2, 64, edge_maps=True)
    ens.advance(2)
    ens.set_shapes(4, 256)
    ens.advance(2)
    ens.set_shapes(0)
    ens.advance(2)
    for s in (a, b):
        assert rel_l2(s.force_history(8), fa) < 1e-12
    with pytest.raises(ib.IbgError):
        ens.set_shapes(3, 128)
    ens.close()
    for s in (alone, a, b):
        s.close()
