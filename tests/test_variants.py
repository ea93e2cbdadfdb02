"""The other N(x) forms of the reference on the GPU (src/IBSolver.cc:211-283):
LinearizedIBSolver, LinearizedPeriodicIBSolver, AdjointIBSolver and SFDSolver, against fixtures
the reference itself produced (tests/golden/var_*.npz, made by
tests/golden/make_golden.py), to the FP64 parity bar."""
import numpy as np
import pytest

from helpers import FP64_TOL, load_golden, rel_l2, variant_names


def _solver(d):
    import ibpm_b200 as ib
    grid = ib.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
                   float(d["yoffset"]))
    geo = ib.geometry.parse(str(d["geom"]))
    model_name = str(d["model"])
    linear = model_name in ("linear", "linearperiodic", "adjoint")
    # the linear models run without the uniform base flow, as the reference CLI builds them
    model = ib.NavierStokesModel(grid, geo, float(d["Re"]), u_mag=0.0 if linear else 1.0)
    s = ib.NonlinearIBSolver(grid, model, float(d["dt"]), str(d["scheme"]), float(d["tol"]))
    if model_name == "adjoint":
        s.set_adjoint(d["base_omega"][0], d["base_q"][0])
    elif linear:
        P = int(d["period"])
        s.set_linearized([d["base_omega"][k] for k in range(P)], [d["base_q"][k] for k in range(P)])
    else:
        s.set_sfd(float(d["chi"]), float(d["Delta"]), np.zeros(grid.scalar().shape))
    return ib, grid, geo, s


@pytest.mark.gpu
@pytest.mark.parametrize("name", variant_names())
def test_gpu_variant_matches_reference(name):
    d = load_golden(name)
    ib, grid, geo, s = _solver(d)
    s.init()
    x = ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float))
    s.set_state(x, with_q=False)
    n = int(d["nsteps"])
    s.advance_resident(n)          # the first step runs eagerly, the others as the captured graph
    forces = s.force_history(n)
    s.get_state(x)
    assert rel_l2(forces, d["forces"][:, 2:4]) < FP64_TOL
    assert rel_l2(x.omega, d["omega"]) < FP64_TOL
    assert rel_l2(x.q, d["q"]) < FP64_TOL
    s.close()


@pytest.mark.gpu
def test_gpu_sfd_filtered_state_and_switching_back():
    """The filtered state follows the oracle's; period 0 restores the nonlinear N(x)."""
    from helpers import oracle_from_variant
    d = load_golden("var_sfd_l2_rk3")
    ib, grid, geo, s = _solver(d)
    s.init()
    s.set_state(ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float)), with_q=False)
    s.advance_resident(3)
    g, model, so, xo = oracle_from_variant(d)
    model.update_operators(xo.time)
    xo.q = model.flux(xo.omega)
    so.init()
    for _ in range(3):
        so.advance(xo)
    assert rel_l2(s.sfd_filtered(), so.sfd["what"]) < FP64_TOL
    s.set_linearized(None)
    with pytest.raises(ib.IbgError):
        s.sfd_filtered()
    s.close()
