"""The CPU oracle (numpy restatement) against the reference.

* every golden fixture (generated from the reference library itself by
  tests/golden/make_golden.py) is reproduced by the restatement;
* when oracle/_ref is built (the reference sources compiled with the FFTW
  shim), each hot-path operator of the restatement is compared with the
  reference's own operator on random inputs.
"""
import numpy as np
import pytest

from helpers import FP64_TOL, golden_names, load_golden, oracle_from_golden, rel_l2
from oracle import ibpm_oracle as O
from oracle import refops as R

needs_ref = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (needs the reference sources)")


@pytest.mark.parametrize("name", golden_names())
def test_oracle_reproduces_golden(name):
    d = load_golden(name)
    g, model, solver, x = oracle_from_golden(d)
    model.update_operators(x.time)
    x.q = model.flux(x.omega)
    solver.init()
    forces = []
    for _ in range(int(d["nsteps"])):
        solver.advance(x)
        forces.append(x.net_force())
    assert rel_l2(np.array(forces), d["forces"][:, 2:4]) < FP64_TOL
    assert rel_l2(x.omega, d["omega"]) < FP64_TOL
    assert rel_l2(x.q, d["q"]) < FP64_TOL
    assert rel_l2(x.f, d["f"]) < 1e-9
    assert x.timestep == int(d["timestep"])


def test_dst1_matches_scipy():
    from scipy.fft import dst
    rng = np.random.default_rng(0)
    for n in (1, 3, 7, 199, 255):
        x = rng.standard_normal((3, n))
        assert np.allclose(O.dst1(x, -1), dst(x, type=1, axis=-1), rtol=1e-12, atol=1e-12)


GRIDS = [(8, 12, 3, 1.3, -0.4, -0.5), (16, 16, 2, 2.0, -1.0, -1.0), (12, 20, 1, 1.0, 0.0, 0.0),
         (32, 16, 4, 3.0, -1.0, -0.5)]


@needs_ref
def test_shim_dst_matches_scipy():
    from scipy.fft import dst
    rng = np.random.default_rng(1)
    for shape in ((7, 11), (1, 5), (199, 13), (30, 22)):
        x = rng.standard_normal(shape)
        ref = dst(dst(x, type=1, axis=0), type=1, axis=1)
        assert np.abs(R.dst2d(x) - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())


@needs_ref
@pytest.mark.parametrize("gp", GRIDS)
def test_operators_match_reference(gp):
    g = O.Grid(*gp)
    rng = np.random.default_rng(sum(gp[:3]))
    s = rng.standard_normal(g.scalar().shape)
    q = rng.standard_normal(g.flux().shape)

    def same(a, b, tol=0.0):
        m = ~np.isnan(b)
        assert np.array_equal(np.isnan(a), np.isnan(b))
        err = np.abs(a[m] - b[m]).max() / max(1.0, np.abs(b[m]).max())
        assert err <= tol, err

    same(O.coarsify(g, s), R.coarsify(g, s))
    for lev in range(g.ngrid - 1):
        same(O.bc_ring(g, O.get_bc(g, s, lev)), R.getbc_ring(g, s, lev))
    same(O.curl_flux(g, q), R.curl_flux(g, q))
    same(O.curl_scalar(g, s), R.curl_scalar(g, s))
    same(O.laplacian(g, s), R.laplacian(g, s))
    u, v = R.flux_to_velocity(g, q)
    same(O.flux_to_xvel(g, q), u)
    same(O.flux_to_yvel(g, q), v)
    qo = g.flux()
    O.xvel_to_flux(g, u, qo)
    O.yvel_to_flux(g, v, qo)
    same(qo, R.velocity_to_flux(g, u, v))
    same(O.cross_product(g, q, s), R.cross_product(g, q, s))
    same(O.nonlinear(g, q, s), R.nonlinear(g, q, s))
    same(O.EllipticSolver(g, "poisson").solve(s), R.elliptic(g, "poisson", 0.0, s), 1e-13)
    same(O.EllipticSolver(g, "helmholtz", -0.013).solve(s), R.elliptic(g, "helmholtz", -0.013, s), 1e-13)


@needs_ref
def test_regularizer_projection_match_reference():
    rng = np.random.default_rng(3)
    g = O.Grid(32, 32, 2, 2.0, -1.0, -1.0)
    xy = O.circle_points(0.05, -0.02, 0.3, 21)
    reg = O.Regularizer(g)
    reg.update(xy)
    f = rng.standard_normal(42)
    q = rng.standard_normal(g.flux().shape)
    assert np.array_equal(reg.to_flux(f), R.reg_toflux(g, xy, f))
    assert np.array_equal(reg.to_boundary(q), R.reg_toboundary(g, xy, q))
    model = O.Model(g, [O.Body(xy)], Re=100.0)
    ps = O.ProjectionSolver(model, 0.01)
    assert rel_l2(ps.M(f), R.apply_m(g, xy, 100.0, 0.01, f)) < 1e-13
    ps.init()
    a = rng.standard_normal(g.scalar().shape)
    b = rng.standard_normal(42)
    w, ff = ps.solve(a, b, np.zeros(42))
    wr, fr = R.projection(g, xy, 100.0, 0.01, a, b, np.zeros(42))
    assert rel_l2(w, wr) < 1e-12 and rel_l2(ff, fr) < 1e-12
    cg = O.ProjectionSolver(model, 0.01, "cg", 1e-10)
    w2, f2 = cg.solve(a, b, np.zeros(42))
    wr2, fr2 = R.projection(g, xy, 100.0, 0.01, a, b, np.zeros(42), use_cg=True, tol=1e-10)
    assert rel_l2(w2, wr2) < 1e-12 and rel_l2(f2, fr2) < 1e-12


def test_restart_roundtrip(tmp_path):
    g = O.Grid(16, 8, 2, 2.0, -1.0, -0.5)
    rng = np.random.default_rng(4)
    x = O.State(g, 5, omega=rng.standard_normal(g.scalar().shape), q=rng.standard_normal(g.flux().shape),
                f=rng.standard_normal(10), timestep=7, time=0.125)
    p = str(tmp_path / "r.bin")
    O.save_restart(p, x, g)
    d = O.load_restart(p)
    assert d["nx"] == 16 and d["ny"] == 8 and d["ngrid"] == 2 and d["npts"] == 5
    assert np.array_equal(d["omega"], x.omega) and np.array_equal(d["q"], x.q) and np.array_equal(d["f"], x.f)
    assert d["timestep"] == 7 and d["time"] == 0.125


@pytest.mark.parametrize("name", __import__("helpers").variant_names())
def test_oracle_reproduces_variant_golden(name):
    """Linearized, linearized-periodic and SFD solvers (src/IBSolver.cc:211-283) against
    fixtures the reference itself produced."""
    from helpers import oracle_from_variant
    d = load_golden(name)
    g, model, solver, x = oracle_from_variant(d)
    model.update_operators(x.time)
    x.q = model.flux(x.omega)
    solver.init()
    forces = []
    for _ in range(int(d["nsteps"])):
        solver.advance(x)
        forces.append(x.net_force())
    assert rel_l2(np.array(forces), d["forces"][:, 2:4]) < FP64_TOL
    assert rel_l2(x.omega, d["omega"]) < FP64_TOL
    assert rel_l2(x.q, d["q"]) < FP64_TOL
