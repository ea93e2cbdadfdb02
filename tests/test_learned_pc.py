"""Learned preconditioner of the moving-body force solve.

CPU: the oracle's hand-written backward against central finite differences.
GPU: the CUDA training kernels' loss and gradient against the oracle, the
BF16 inference against the oracle's forward, and a trained network cutting
the flexible-PCG iterations of the pitching plate below plain CG at the same
absolute tolerance while the forces stay those of the reference.
"""
import numpy as np
import pytest

from helpers import load_golden, rel_l2
from oracle import learned_pc as LP


def _tiny_case(seed=0, B=2):
    rng = np.random.default_rng(seed)
    th = np.linspace(0, 2 * np.pi, 5, endpoint=False)
    circle = np.stack([np.cos(th), np.sin(th)], 1)
    line = np.stack([np.linspace(-0.5, 0.5, 3), np.zeros(3)], 1)
    nbr, cnt = LP.neighbours([circle, line])
    P = len(cnt)
    geom = rng.standard_normal((B, P, 4))
    A = rng.standard_normal((B, 2 * P, 2 * P))
    mb = A @ A.transpose(0, 2, 1) / (2 * P) + np.eye(2 * P)
    p = rng.standard_normal(LP.N_PARAMS) * 0.2
    p[LP.O_C0] = 1.7
    return p, geom, mb, nbr, cnt


def test_neighbour_lists():
    th = np.linspace(0, 2 * np.pi, 10, endpoint=False)
    nbr, cnt = LP.neighbours([np.stack([np.cos(th), np.sin(th)], 1), np.stack([np.arange(3.0), np.zeros(3)], 1)])
    assert list(cnt[:10]) == [8] * 10 and list(cnt[10:]) == [2, 2, 2]
    assert sorted(nbr[0][:8]) == [1, 2, 3, 4, 6, 7, 8, 9]
    assert sorted(nbr[10][:2]) == [11, 12]
    # symmetric with multiplicity (the backward relies on it)
    P = len(cnt)
    Mx = np.zeros((P, P), int)
    for i in range(P):
        for q in range(cnt[i]):
            Mx[i, nbr[i, q]] += 1
    assert (Mx == Mx.T).all()


def test_oracle_gradient_matches_finite_differences():
    p, geom, mb, nbr, cnt = _tiny_case()
    loss, g = LP.loss_grad(p, geom, mb, nbr, cnt)
    rng = np.random.default_rng(1)
    blocks = [(LP.O_W1, LP.O_B1), (LP.O_B1, LP.O_W2), (LP.O_W2, LP.O_B2), (LP.O_B2, LP.O_W3), (LP.O_W3, LP.O_B3),
              (LP.O_B3, LP.O_C0)]
    h = 1e-6
    f = lambda q: LP.loss_grad(q, geom, mb, nbr, cnt)[0]
    for a, b in blocks:
        for k in rng.integers(a, b, size=min(5, b - a)):
            pp, pm = p.copy(), p.copy()
            pp[k] += h
            pm[k] -= h
            fd = (f(pp) - f(pm)) / (2 * h)
            assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-8, (k, fd, g[k])
    d = rng.standard_normal(LP.N_PARAMS)
    d[LP.O_C0] = 0.0
    fd = (f(p + h * d) - f(p - h * d)) / (2 * h)
    assert abs(fd - g @ d) < 1e-5 * max(1.0, abs(fd))
    assert g[LP.O_C0] == 0.0 and loss > 0


def test_oracle_operator_is_symmetric_and_scaled():
    p, geom, mb, nbr, cnt = _tiny_case(B=1)
    K1 = LP.operator(p, geom[0], nbr, cnt, 0.5)
    K2 = LP.operator(p, geom[0], nbr, cnt, 0.25)
    assert np.allclose(K1, K1.T)
    assert np.allclose(K2, 2.0 * K1)


def _plate():
    import ibpm_b200 as ib
    d = load_golden("plate_l2_pitchplunge_cg")
    grid = ib.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
                   float(d["yoffset"]))
    geo = ib.geometry.parse(str(d["geom"]))
    return ib, d, grid, geo


def _nbr_of(geo):
    return LP.neighbours([np.array(b.points, dtype=float) for b in geo.bodies])


@pytest.mark.gpu
def test_gpu_loss_and_gradient_match_oracle():
    """The FP32 forward/backward kernels against the float64 restatement, on
    operators the solver generates for the pitching plate."""
    ib, d, grid, geo = _plate()
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, float(d["Re"])), float(d["dt"]), "rk3",
                             float(d["tol"]), precond="learned")
    geom, mb = s.lpc_generate(3, 0.0, 2.0)
    assert np.isfinite(geom).all() and np.isfinite(mb).all()
    m = mb.shape[1]
    # M / beta is nearly symmetric and positive definite
    assert rel_l2(mb, mb.transpose(0, 2, 1)) < 1e-3
    assert min(np.linalg.eigvalsh(0.5 * (x + x.T)).min() for x in mb) > 0
    nbr, cnt = _nbr_of(geo)
    p = s.lpc_params()
    p[LP.O_C0] = float(np.mean([np.trace(x) for x in mb]) / m)
    loss_gpu, g_gpu = s.lpc_loss_grad(geom, mb, params=p)
    loss_cpu, g_cpu = LP.loss_grad(p, geom, mb, nbr, cnt)
    assert abs(loss_gpu - loss_cpu) < 1e-4 * loss_cpu
    for a, b in ((LP.O_W1, LP.O_B1), (LP.O_B1, LP.O_W2), (LP.O_W2, LP.O_B2), (LP.O_B2, LP.O_W3),
                 (LP.O_W3, LP.O_B3), (LP.O_B3, LP.O_C0)):
        assert rel_l2(g_gpu[a:b], g_cpu[a:b]) < 1e-3, (a, b)
    assert g_gpu[LP.O_C0] == 0.0
    s.close()


@pytest.mark.gpu
def test_gpu_training_lowers_loss_and_pcg_iterations():
    """Train on the plate's own force operators, then advance: the forces match
    the reference at the same absolute CG tolerance, with at most 0.8 times the
    iterations of plain CG; the BF16 inference agrees with the float64 forward."""
    ib, d, grid, geo = _plate()
    model = ib.NavierStokesModel(grid, geo, float(d["Re"]))
    n = int(d["nsteps"])
    its = {}
    for pc in ("none", "learned"):
        s = ib.NonlinearIBSolver(grid, model, float(d["dt"]), "rk3", float(d["tol"]), precond=pc)
        x = ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float))
        if pc == "learned":
            geom, mb = s.lpc_generate(16, 0.0, 4.0)
            hist = s.lpc_train(geom, mb, epochs=150, batch=4, lr=1e-3, seed=1)
            assert hist[-1] < 0.3 * hist[0], hist
            nbr, cnt = _nbr_of(geo)
            r = np.random.default_rng(2).standard_normal(2 * geo.num_points)
            z, gm = s.lpc_apply(0, r)
            zc = LP.operator(s.lpc_params(), gm, nbr, cnt, s.beta(0)) @ r
            assert rel_l2(z, zc) < 3e-2
        s.init()
        s.set_state(x, with_q=False)
        s.advance_resident(n)
        forces = s.force_history(n)
        s.get_state(x)
        its[pc] = s.cg_totals()[0]
        assert rel_l2(forces, d["forces"][:, 2:4]) < 1e-8
        assert rel_l2(x.omega, d["omega"]) < 1e-9
        s.close()
    # measured on the B200: 791 against 1246 iterations over the run (0.63)
    assert its["learned"] < 0.8 * its["none"], its


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["plate", "two_cylinders_402"])
def test_tensor_core_inference_matches_cuda_cores_and_oracle(case):
    """The network's 256 x 256 layer on tcgen05 (the default) against the same
    evaluation on the CUDA cores and against the float64 forward: both use BF16
    weights and activations with FP32 accumulation, so they agree to BF16
    rounding.  The two-cylinder case has 402 points (161,604 pairs, 1263 tiles of
    128 pairs over the persistent CTAs)."""
    import ctypes
    import ibpm_b200 as ib
    from ibpm_b200 import _native, configs
    if case == "plate":
        ib, d, grid, geo = _plate()
        s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, float(d["Re"])), float(d["dt"]), "rk3",
                                 float(d["tol"]), precond="learned")
    else:
        wl = configs.c5_two_cylinders()
        grid = ib.Grid(128, 128, 1, 4.0, -2.0, -2.0)
        geo = ib.geometry.parse(wl.geom)
        s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, wl.Re), wl.dt, "rk3", 1e-7,
                                 precond="learned")
    L = _native.lib()
    rng = np.random.default_rng(3)
    p = s.lpc_params()
    p[:-1] += 0.05 * rng.standard_normal(p.size - 1)  # away from the initialisation, as after training
    p[LP.O_C0] = 2.5
    s.lpc_set_params(p)
    r = rng.standard_normal(2 * geo.num_points)
    z_tc, gm = s.lpc_apply(0, r)
    assert L.ibg_lpc_status(s.handle) == 0
    assert L.ibg_lpc_set_tensor_cores(s.handle, 0) == 0
    z_cc, _ = s.lpc_apply(0, r)
    assert L.ibg_lpc_set_tensor_cores(s.handle, 1) == 0
    nbr, cnt = _nbr_of(geo)
    zc = LP.operator(s.lpc_params(), gm, nbr, cnt, s.beta(0)) @ r
    assert rel_l2(z_tc, z_cc) < 1e-2, rel_l2(z_tc, z_cc)
    assert rel_l2(z_tc, zc) < 3e-2
    assert rel_l2(z_cc, zc) < 3e-2
    # twice in a row gives the same result (the persistent CTAs hold no state between calls)
    z_tc2, _ = s.lpc_apply(0, r)
    assert np.array_equal(z_tc, z_tc2)
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("fallback_iter", [0, 20])
def test_a_useless_network_still_gives_the_references_forces(fallback_iter):
    """A network with random weights: the flexible PCG falls back to plain CG (when r.z <= 0, or after
    pc_fallback_iter iterations; 0 = a quarter of the iteration cap) and the solve still converges to
    the reference's tolerance, no solve stopping at the cap."""
    ib, d, grid, geo = _plate()
    model = ib.NavierStokesModel(grid, geo, float(d["Re"]))
    n = int(d["nsteps"])
    s = ib.NonlinearIBSolver(grid, model, float(d["dt"]), "rk3", float(d["tol"]), precond="learned",
                             pc_fallback_iter=fallback_iter)
    p = s.lpc_params()
    rng = np.random.default_rng(7)
    p[:-1] = rng.standard_normal(len(p) - 1).astype(p.dtype) * 0.5
    p[-1] = 1.0  # the operator scale c0
    s.lpc_set_params(p)
    x = ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float))
    s.init()
    s.set_state(x, with_q=False)
    s.advance_resident(n)
    forces = s.force_history(n)
    _, _, capped = s.cg_stats()
    assert capped == 0
    assert rel_l2(forces, d["forces"][:, 2:4]) < 1e-8
    s.close()
