"""The kernel-launch counts the library reports (per step, per ensemble step)
against the kernel nodes of the CUDA graphs it captured.

bench.py's `gpu_launches` is the library's own count; these tests check that
count against the graph itself for fixed-body contexts in FP64 and FP32, one
and several levels, RK3 and AB2, and for an ensemble whose members run the
fused sweep (the per-step line FFTs inside the sums launch).
"""
import pytest

pytestmark = pytest.mark.gpu


def _solver(gp, precision="fp64", scheme="rk3"):
    import ibpm_b200 as ib
    from ibpm_b200 import configs, geometry
    grid = ib.Grid(*gp)
    geo = geometry.parse(configs.cylinder_geom(24, r=0.1 * gp[3]))
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, 100.0), 0.01, scheme, precision=precision)
    x = ib.State(grid, s.npoints)
    s.init()
    s.set_state(x, with_q=False)
    return s


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("gp,scheme", [((64, 64, 1, 2.0, -1.0, -1.0), "rk3"),
                                       ((96, 64, 3, 3.0, -1.5, -1.0), "rk3"),
                                       ((64, 48, 2, 2.0, -1.0, -0.75), "ab2")])
def test_step_graph_kernel_nodes_match_the_reported_launches(gp, scheme, precision):
    from ibpm_b200 import _native
    L = _native.lib()
    s = _solver(gp, precision, scheme)
    s.advance_resident(3)  # the first step runs unrecorded; the next ones launch the step graph
    nodes = L.ibg_graph_kernel_nodes(s.handle)
    claim = L.ibg_graph_launch_claim(s.handle)
    assert nodes > 0
    assert nodes == claim, (nodes, claim)
    assert s.last_launch_count() == 3 * claim  # the first step, run directly, counts the same kernels
    s.advance_resident(1)
    assert s.last_launch_count() == claim
    s.close()


def test_ensemble_graph_kernel_nodes_match_the_reported_launches():
    import ibpm_b200 as ib
    from ibpm_b200 import _native
    L = _native.lib()
    members = [_solver((64, 64, 3, 2.0, -1.0, -1.0), "fp32"), _solver((96, 96, 2, 3.0, -1.5, -1.5), "fp32"),
               _solver((64, 64, 1, 2.0, -1.0, -1.0), "fp64")]
    for m in members:
        m.advance_resident(1)
    ens = ib.Ensemble(members)
    ens.advance(2)
    nodes = L.ibg_ensemble_kernel_nodes(ens._h)
    assert nodes > 0
    assert nodes == ens.launches_per_step(), (nodes, ens.launches_per_step())
    ens.close()
    for m in members:
        m.close()
