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


def _tiny_case(seed=0, B=3):
    rng = np.random.default_rng(seed)
    th = np.linspace(0, 2 * np.pi, 13, endpoint=False)
    circle = np.stack([np.cos(th), np.sin(th)], 1)
    line = np.stack([np.linspace(-0.5, 0.5, 6), np.zeros(6)], 1)
    nbr, cnt = LP.neighbours([circle, line])
    P = len(cnt)
    geom = rng.standard_normal((B, P, 4))
    r = rng.standard_normal((B, 2 * P))
    zb = rng.standard_normal((B, 2 * P))
    p = rng.standard_normal(LP.N_PARAMS) * 0.2
    return p, geom, r, zb, nbr, cnt


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
    p, geom, r, zb, nbr, cnt = _tiny_case()
    loss, g = LP.loss_grad(p, geom, r, zb, nbr, cnt)
    rng = np.random.default_rng(1)
    # a sample of coordinates from every parameter block
    blocks = [(LP.O_W1, LP.O_B1), (LP.O_B1, LP.O_W2), (LP.O_W2, LP.O_B2), (LP.O_B2, LP.O_W3), (LP.O_W3, LP.O_B3),
              (LP.O_B3, LP.N_PARAMS)]
    h = 1e-6
    for a, b in blocks:
        for k in rng.integers(a, b, size=min(6, b - a)):
            pp, pm = p.copy(), p.copy()
            pp[k] += h
            pm[k] -= h
            fd = (LP.loss_grad(pp, geom, r, zb, nbr, cnt)[0] - LP.loss_grad(pm, geom, r, zb, nbr, cnt)[0]) / (2 * h)
            assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-8, (k, fd, g[k])
    # directional derivative along a random direction
    d = rng.standard_normal(LP.N_PARAMS)
    fd = (LP.loss_grad(p + h * d, geom, r, zb, nbr, cnt)[0] - LP.loss_grad(p - h * d, geom, r, zb, nbr, cnt)[0]) / (2 * h)
    assert abs(fd - g @ d) < 1e-5 * max(1.0, abs(fd))
    assert loss > 0


def test_preconditioner_is_positively_homogeneous():
    p, geom, r, zb, nbr, cnt = _tiny_case(B=1)
    z1 = LP.apply(p, geom[0], r[0], nbr, cnt, 0.5)
    z2 = LP.apply(p, geom[0], 3.0 * r[0], nbr, cnt, 0.5)
    assert rel_l2(z2, 3.0 * z1) < 1e-13


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
    ib, d, grid, geo = _plate()
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, float(d["Re"])), float(d["dt"]), "rk3",
                             float(d["tol"]), precond="learned")
    geom, r, zb = s.lpc_generate(2, 0.0, 1.0, 3, seed=5)
    assert np.isfinite(geom).all() and np.isfinite(zb).all() and np.abs(zb).max() > 0
    nbr, cnt = _nbr_of(geo)
    p = s.lpc_params()
    loss_gpu, g_gpu = s.lpc_loss_grad(geom, r, zb)
    loss_cpu, g_cpu = LP.loss_grad(p, geom, r, zb, nbr, cnt)
    # FP32 kernels against the float64 restatement
    assert abs(loss_gpu - loss_cpu) < 1e-5 * loss_cpu
    assert rel_l2(g_gpu, g_cpu) < 1e-4
    for a, b in ((LP.O_W1, LP.O_B1), (LP.O_W2, LP.O_B2), (LP.O_W3, LP.O_B3), (LP.O_B1, LP.O_W2)):
        assert rel_l2(g_gpu[a:b], g_cpu[a:b]) < 1e-4
    # explicit parameters replace the current ones
    p2 = p * 0.5
    loss2, g2 = s.lpc_loss_grad(geom, r, zb, params=p2)
    assert abs(loss2 - LP.loss_grad(p2, geom, r, zb, nbr, cnt)[0]) < 1e-5 * loss2
    s.close()


@pytest.mark.gpu
def test_gpu_training_lowers_loss_and_pcg_iterations():
    """Train on the plate's own force operator, then advance: forces match the
    reference at the same absolute tolerance, with fewer CG iterations."""
    ib, d, grid, geo = _plate()
    model = ib.NavierStokesModel(grid, geo, float(d["Re"]))
    n = int(d["nsteps"])
    its = {}
    for pc in ("none", "learned"):
        s = ib.NonlinearIBSolver(grid, model, float(d["dt"]), "rk3", float(d["tol"]), precond=pc)
        x = ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float))
        if pc == "learned":
            geom, r, zb = s.lpc_generate(8, 0.0, n * float(d["dt"]), 32, seed=3)
            hist = s.lpc_train(geom, r, zb, epochs=60, batch=32, lr=1e-3, seed=1)
            assert hist[-1] < 0.5 * hist[0], hist
            # BF16 inference on the device against the float64 forward of the trained weights
            nbr, cnt = _nbr_of(geo)
            rr = r[5].astype(np.float64)
            z, gm = s.lpc_apply(0, rr)
            zc = LP.apply(s.lpc_params(), gm, rr, nbr, cnt, s.beta(0))
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
    assert its["learned"] < its["none"], its
