"""The allocation-free Poisson entry point against the context-based one.

ibg_poisson_solve_static exists for callers that cannot call cudaMalloc (for
example code running inside a graph capture into a pool it does not own, or a
plug-in whose host application forbids device allocation).  It keeps its
scratch and its per-shape tables in fixed file-scope device arrays, so these
tests check that calls in a row (each finding the previous call's scratch
contents) agree with ibg_poisson_solve, also when the grid shape changes and a
table slot is reused, that repeated calls leave the device's free memory
unchanged, that a grid too large for the arrays is refused, and that a call
that would upload tables during a stream capture is refused.  The tests
allocate their own input and output buffers; the entry point does not.
"""
import ctypes

import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the operator tolerance of the other GPU parity tests


def _context(gp):
    import ibpm_b200 as ib
    from ibpm_b200 import geometry
    grid = ib.Grid(*gp)
    geo = geometry.Geometry([geometry.RigidBody(points=[(0.0, 0.0), (0.1, 0.0)])])
    return grid, ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, 100.0), 0.01, "rk3")


def _static(gp, f_dev, u_dev, stream):
    from ibpm_b200 import _native
    L = _native.lib()
    g = _native.ibg_grid(*gp)
    return L.ibg_poisson_solve_static(ctypes.byref(g), ctypes.c_void_p(f_dev.data_ptr()),
                                      ctypes.c_void_p(u_dev.data_ptr()), ctypes.c_void_p(stream))


def test_static_poisson_matches_context_poisson_twice():
    import torch
    from ibpm_b200 import _native
    gp = (128, 64, 3, 4.0, -2.0, -1.0)
    grid, solver = _context(gp)
    rng = np.random.default_rng(11)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        f = rng.standard_normal(grid.scalar().shape)
        expected = solver.poisson(f)
        f_dev = torch.from_numpy(f).cuda()
        u_dev = torch.full_like(f_dev, float("nan"))
        st = _static(gp, f_dev, u_dev, stream)
        assert st == 0, _native.lib().ibg_static_last_error()
        torch.cuda.synchronize()
        assert rel_l2(u_dev.cpu().numpy(), expected) < TOL, f"call {call}"
    solver.close()


def test_static_poisson_alternating_shapes():
    """Shape changes on one stream: A, B, A, then three more shapes so that a
    fifth shape replaces the least recently used table slot, then A again."""
    import torch
    from ibpm_b200 import _native
    shapes = [(128, 64, 3, 4.0, -2.0, -1.0), (96, 64, 3, 3.0, -1.5, -1.0), (64, 96, 2, 2.0, -1.0, -1.5),
              (80, 48, 2, 2.5, -1.25, -0.75), (160, 32, 1, 5.0, -2.5, -0.5), (45, 27, 1, 3.0, -1.5, -0.9)]
    order = [0, 1, 0, 2, 3, 4, 1, 0, 5, 3]  # (the last shape has odd sizes: odd half-length DSTs)
    ctxs = [_context(gp) for gp in shapes]
    rng = np.random.default_rng(12)
    stream = torch.cuda.current_stream().cuda_stream
    for call, k in enumerate(order):
        grid, solver = ctxs[k]
        f = rng.standard_normal(grid.scalar().shape)
        expected = solver.poisson(f)
        f_dev = torch.from_numpy(f).cuda()
        u_dev = torch.full_like(f_dev, float("nan"))
        st = _static(shapes[k], f_dev, u_dev, stream)
        assert st == 0, _native.lib().ibg_static_last_error()
        torch.cuda.synchronize()
        assert rel_l2(u_dev.cpu().numpy(), expected) < TOL, f"call {call} shape {shapes[k][:3]}"
    for _, s in ctxs:
        s.close()


def test_static_poisson_allocates_nothing():
    """After one call per shape (which may load the library's device module,
    whose static arrays are the entry point's memory), further calls with
    alternating shapes leave the device's free memory unchanged."""
    import torch
    from ibpm_b200 import _native
    shapes = [(128, 64, 3, 4.0, -2.0, -1.0), (96, 64, 3, 3.0, -1.5, -1.0)]
    stream = torch.cuda.current_stream().cuda_stream
    bufs = []
    for gp in shapes:
        n = gp[2] * (gp[0] - 1) * (gp[1] - 1)
        bufs.append((torch.randn(n, dtype=torch.float64, device="cuda"),
                     torch.empty(n, dtype=torch.float64, device="cuda")))
    for gp, (f_dev, u_dev) in zip(shapes, bufs):
        assert _static(gp, f_dev, u_dev, stream) == 0, _native.lib().ibg_static_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k in (0, 1, 0, 1, 1, 0):
        assert _static(shapes[k], bufs[k][0], bufs[k][1], stream) == 0, _native.lib().ibg_static_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"


def test_static_poisson_refuses_table_upload_during_capture():
    import torch
    from ibpm_b200 import _native
    gp = (112, 48, 2, 3.5, -1.75, -0.75)  # a shape no other test uses: its tables are not loaded
    f_dev = torch.zeros(2 * 111 * 47, dtype=torch.float64, device="cuda")
    u_dev = torch.zeros_like(f_dev)
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        st = _static(gp, f_dev, u_dev, s.cuda_stream)
        g.capture_end()
    assert st < 0
    assert b"captur" in _native.lib().ibg_static_last_error()


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
