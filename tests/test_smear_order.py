"""The regularizer smear's fixed-order gather, restated on the CPU against the reference's order.

The reference smears boundary forces onto level-0 fluxes by walking its association list, built
direction by direction, point by point, flux index by flux index (src/Regularizer.cc:54-109), adding
each weight x force into its flux in that order.  The GPU smear has no atomics
(ibpm_b200/csrc/ops.cu, k_reg_owners / k_reg_smear): each (component, slot) looks for the other
components of the same direction that hold the same flux -- searching only the points within 3.5 cells
in x and in y -- and the first of them in component order writes the sum over all of them, in component
order.  These tests check, without a GPU, that (a) the 3.5-cell window finds every component that
shares a flux (each point's support reaches under 1.5 cells, so sharers are under 3 cells apart), (b)
no component holds more than the 16 slots the kernels keep, and (c) the owners' sums equal the
reference-ordered accumulation bit for bit.
"""
import numpy as np
import pytest

from oracle import ibpm_oracle as O

K_SLOTS = 16


def _bodies(kind, g, rng):
    h = g.dx
    if kind == "cylinder":
        n = int(round(2 * np.pi * 0.3 / h))
        t = 2 * np.pi * np.arange(n) / n
        return np.stack([0.3 * np.cos(t) + 0.01, 0.3 * np.sin(t) - 0.02], 1)
    if kind == "dense_cylinder":  # points a quarter cell apart: many components per flux
        n = int(round(2 * np.pi * 0.2 / (0.25 * h)))
        t = 2 * np.pi * np.arange(n) / n
        return np.stack([0.2 * np.cos(t), 0.2 * np.sin(t)], 1)
    if kind == "two_plates":  # crossing plates and a second body close by
        s = np.linspace(-0.4, 0.4, int(0.8 / h) + 1)
        a = np.stack([s, 0.3 * s + 0.003], 1)
        b = np.stack([-0.5 * s + 0.004, s], 1)
        c = np.stack([s * 0.5 + 0.1, np.full_like(s, 0.05 + 0.5 * h)], 1)
        return np.concatenate([a, b, c])
    return rng.uniform(-0.6, 0.6, size=(300, 2))  # a random cloud


def _slots(reg, ncomp):
    """Per component: its flux indices (ascending) and weights, as the kernels' slots hold them."""
    idx = [[] for _ in range(ncomp)]
    w = [[] for _ in range(ncomp)]
    for fi, c, wt in zip(reg.flux_idx, reg.bnd_idx, reg.weight):
        idx[c].append(int(fi))
        w[c].append(float(wt))
    return idx, w


@pytest.mark.parametrize("kind", ["cylinder", "dense_cylinder", "two_plates", "cloud"])
def test_owner_sums_match_the_reference_order(kind):
    g = O.Grid(64, 64, 1, 2.0, -1.0, -1.0)
    rng = np.random.default_rng(5)
    pts = _bodies(kind, g, rng)
    npts = pts.shape[0]
    ncomp = 2 * npts
    reg = O.Regularizer(g)
    reg.update(pts)
    idx, w = _slots(reg, ncomp)
    assert max(len(s) for s in idx) <= K_SLOTS
    h, lim = g.dx, 3.5 * g.dx
    f = rng.standard_normal(ncomp)

    # the reference's order: walk the association list, add into each flux in turn
    ref = np.zeros(g.n_flux)
    for fi, c, wt in zip(reg.flux_idx, reg.bnd_idx, reg.weight):
        ref[fi] = ref[fi] + wt * f[c]

    # (a) every pair of components sharing a flux is within the search window
    holders = {}
    for c in range(ncomp):
        for j in idx[c]:
            holders.setdefault(j, []).append(c)
    for j, cs in holders.items():
        for c1 in cs:
            for c2 in cs:
                p1, p2 = c1 % npts, c2 % npts
                assert c1 // npts == c2 // npts  # x and y fluxes never share an index
                assert abs(pts[p1, 0] - pts[p2, 0]) <= lim and abs(pts[p1, 1] - pts[p2, 1]) <= lim

    # (c) the kernels' owners, restated: search the window in point order, sum in component order
    got = np.zeros(g.n_flux)
    written = set()
    for c in range(ncomp):
        d, p = divmod(c, npts)
        for j in idx[c]:
            owner, terms = True, []
            for q in range(npts):
                if abs(pts[q, 0] - pts[p, 0]) > lim or abs(pts[q, 1] - pts[p, 1]) > lim:
                    continue
                c2 = d * npts + q
                if j in idx[c2]:
                    if c2 < c:
                        owner = False
                        break
                    terms.append(w[c2][idx[c2].index(j)] * f[c2])
            if not owner:
                continue
            assert j not in written  # one owner per flux
            written.add(j)
            s = 0.0
            for t in terms:
                s = s + t
            got[j] = s
    assert written == set(holders)
    assert np.array_equal(got, ref)
    # and the oracle's smear (np.add.at walks the list in the same order, then times dx) agrees
    assert np.array_equal(reg.to_flux(f)[0], got * h)
