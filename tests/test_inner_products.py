"""Inner products with the reference's multi-domain weights and the energy of
OutputEnergy (src/VectorOperations.cc:222-412, src/OutputEnergy.cc:29-33).

CPU: the oracle's weights against the reference's own InnerProduct /
FineGridInnerProduct (built from its sources).  GPU: the device reductions
against the oracle."""
import numpy as np
import pytest

from helpers import load_golden, rel_l2
from oracle import ibpm_oracle as O
from oracle import refops as R

GRIDS = [(32, 32, 1), (32, 32, 3), (48, 26, 3), (64, 32, 2)]


def _operands(g, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(g.scalar().shape), rng.standard_normal(g.scalar().shape),
            rng.standard_normal(g.flux().shape), rng.standard_normal(g.flux().shape))


@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("nx,ny,L", GRIDS)
def test_oracle_inner_products_match_reference(nx, ny, L):
    g = O.Grid(nx, ny, L, 4.0, -2.0, -1.0)
    a, b, p, q = _operands(g, nx + L)
    for kind, (x, y) in enumerate(((a, b), (a, b), (p, q), (p, q))):
        r = R.inner_product(g, kind, x, y)
        assert abs(O.inner_product(g, kind, x, y) - r) <= 1e-13 * abs(r)


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,L", GRIDS)
def test_gpu_inner_products_match_oracle(nx, ny, L):
    import ibpm_b200 as ib
    from ibpm_b200 import configs
    grid = ib.Grid(nx, ny, L, 4.0, -2.0, -1.0)
    geo = ib.geometry.parse(configs.cylinder_geom(16, r=0.3))
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, 100.0), 0.01, "rk3")
    g = O.Grid(nx, ny, L, 4.0, -2.0, -1.0)
    a, b, p, q = _operands(g, nx + L)
    for fine in (False, True):
        ra = O.inner_product(g, 1 if fine else 0, a, b)
        rp = O.inner_product(g, 3 if fine else 2, p, q)
        assert abs(s.inner_product(a, b, fine_only=fine) - ra) <= 1e-13 * abs(ra)
        assert abs(s.inner_product(p, q, fine_only=fine) - rp) <= 1e-13 * abs(rp)
    s.close()


@pytest.mark.gpu
def test_gpu_energy_of_a_running_state():
    import ibpm_b200 as ib
    d = load_golden("cyl_l3_noise_rk3")
    grid = ib.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
                   float(d["yoffset"]))
    geo = ib.geometry.parse(str(d["geom"]))
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, float(d["Re"])), float(d["dt"]), "rk3")
    s.init()
    x = ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float))
    s.set_state(x, with_q=False)
    s.advance_resident(3)
    e = s.energy()
    s.get_state(x)
    g = O.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
               float(d["yoffset"]))
    ref = 0.5 * O.inner_product(g, 2, x.q, x.q)
    assert abs(e - ref) <= 1e-13 * abs(ref) and e > 0
    s.close()
