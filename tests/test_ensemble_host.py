"""Ensemble.advance_host (ibg_ensemble_advance_host): every member's State copied
in from page-locked host memory, advanced and copied back out, all inside the
ensemble's graph.  The same steps as ibg_ensemble_advance followed by
ibg_get_state, so the same results, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MEMBERS = [((64, 64, 2, 2.0, -1.0, -1.0), "fp32"), ((48, 64, 1, 2.0, -1.0, -1.3), "fp64"),
           ((96, 96, 3, 3.0, -1.5, -1.5), "fp32")]


def _members():
    import ibpm_b200 as ib
    from ibpm_b200 import configs, geometry
    out = []
    for gp, prec in MEMBERS:
        grid = ib.Grid(*gp)
        geo = geometry.parse(configs.cylinder_geom(24, r=0.1 * gp[3]))
        s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, 100.0), 0.01, "rk3", precision=prec)
        x = ib.State(grid, s.npoints)
        s.init()
        s.set_state(x, with_q=False)
        out.append((s, x))
    return out


def _pinned(x):
    import torch
    from types import SimpleNamespace
    h = {}
    for k in ("omega", "q", "f"):
        a = getattr(x, k)
        h[k] = torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()
        h[k][...] = a
    return SimpleNamespace(**h)


def test_advance_host_matches_advance_then_get_state():
    import ibpm_b200 as ib
    ref, host = _members(), _members()
    ens_r = ib.Ensemble([s for s, _ in ref])
    ens_h = ib.Ensemble([s for s, _ in host])
    ens_r.advance(2)
    ens_h.advance(2)
    states = []
    for s, x in host:
        s.get_state(x)
        states.append(_pinned(x))
    for _ in range(3):
        ens_r.advance(1)
        for s, x in ref:
            s.get_state(x)
        ens_h.advance_host(states, 1)
    for (sr, xr), st in zip(ref, states):
        assert np.array_equal(xr.omega, st.omega)
        assert np.array_equal(xr.q, st.q)
        assert np.array_equal(xr.f, st.f)
    for (sr, _), (sh, _) in zip(ref, host):
        assert np.array_equal(sr.force_history(5), sh.force_history(5))
    assert ens_h.host_launches_per_step() == ens_r.launches_per_step() + 4 * 2  # two FP32 members convert
    ens_r.close()
    ens_h.close()
    for s, _ in ref + host:
        s.close()


def test_advance_host_refuses_pageable_arrays():
    import ibpm_b200 as ib
    from types import SimpleNamespace
    members = _members()
    ens = ib.Ensemble([s for s, _ in members])
    ens.advance(1)
    states = [SimpleNamespace(omega=x.omega.copy(), q=x.q.copy(), f=x.f.copy()) for _, x in members]
    with pytest.raises(ib.IbgError):
        ens.advance_host(states, 1)
    ens.close()
    for s, _ in members:
        s.close()


def test_autotune_picks_a_shape_per_grid_class_and_keeps_results():
    """ibg_ensemble_autotune times real ensemble steps per grid class; the shapes it tries compute the
    same butterflies in the same order, so the members' states match an ensemble advanced by as many
    plain steps, bit for bit."""
    import ibpm_b200 as ib
    a, b = _members(), _members()
    ens_a = ib.Ensemble([s for s, _ in a])
    ens_b = ib.Ensemble([s for s, _ in b])
    ens_a.advance(1)
    ens_b.advance(1)
    rows = ens_a.autotune(1)
    assert len(rows) == len({gp[:2] for gp, _ in MEMBERS})
    for r in rows:
        assert (r["pairs_per_cta"], r["threads"]) in {(2, 128), (1, 128), (2, 256), (1, 256), (2, 96)}
        assert r["us_per_step"] > 0
    sa, xa = a[0]
    sa.get_state(xa)
    steps = int(xa.timestep) - 1
    assert steps == (1 + 4 * len(rows)) * 2
    ens_b.advance(steps)
    ens_a.advance(2)
    ens_b.advance(2)
    for (s1, x1), (s2, x2) in zip(a, b):
        s1.get_state(x1)
        s2.get_state(x2)
        assert x1.timestep == x2.timestep
        assert np.array_equal(x1.omega, x2.omega)
        assert np.array_equal(x1.f, x2.f)
    ens_a.close()
    ens_b.close()
    for s, _ in a + b:
        s.close()
