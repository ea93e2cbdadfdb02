"""The allocation-free Poisson entry point against the context-based one.

ibg_poisson_solve_static exists for callers that cannot call cudaMalloc (for
example code running inside a graph capture into a pool it does not own, or a
plug-in whose host application forbids device allocation).  It keeps its
scratch in a fixed file-scope device array, so this test checks that two calls
in a row (the second one finding the first one's scratch contents) both agree
with ibg_poisson_solve, and that a grid too large for the array is refused.
The test allocates its own input and output buffers; the entry point does not.
"""
import ctypes

import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the operator tolerance of the other GPU parity tests


def test_static_poisson_matches_context_poisson_twice():
    import torch
    import ibpm_b200 as ib
    from ibpm_b200 import _native, geometry

    gp = (128, 64, 3, 4.0, -2.0, -1.0)
    grid = ib.Grid(*gp)
    geo = geometry.Geometry([geometry.RigidBody(points=[(0.0, 0.0), (0.1, 0.0)])])
    solver = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, 100.0), 0.01, "rk3")
    rng = np.random.default_rng(11)
    L = _native.lib()
    g = _native.ibg_grid(*gp)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        f = rng.standard_normal(grid.scalar().shape)
        expected = solver.poisson(f)
        f_dev = torch.from_numpy(f).cuda()
        u_dev = torch.full_like(f_dev, float("nan"))
        st = L.ibg_poisson_solve_static(ctypes.byref(g), ctypes.c_void_p(f_dev.data_ptr()),
                                        ctypes.c_void_p(u_dev.data_ptr()), ctypes.c_void_p(stream))
        assert st == 0, L.ibg_static_last_error()
        torch.cuda.synchronize()
        assert rel_l2(u_dev.cpu().numpy(), expected) < TOL, f"call {call}"
    solver.close()


def test_static_poisson_rejects_oversized_grid():
    import torch
    from ibpm_b200 import _native
    L = _native.lib()
    g = _native.ibg_grid(1024, 1024, 2, 16.0, -8.0, -8.0)  # 3 * 1023^2 doubles > 4 MiB
    f_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = L.ibg_poisson_solve_static(ctypes.byref(g), ctypes.c_void_p(f_dev.data_ptr()),
                                    ctypes.c_void_p(f_dev.data_ptr()), None)
    assert st < 0
    assert b"static scratch" in L.ibg_static_last_error()
