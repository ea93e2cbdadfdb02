"""The sine-matrix GEMM form of the FP32 DST passes (dst_gemm.cu: tcgen05
kind::tf32, 3xTF32) against the FFT passes and the FP64 solve.

Both FP32 forms solve to FP32 accuracy against the FP64 multi-domain solve, on
grids whose sizes exercise partial tiles (NI not a multiple of 128, NJ not a
multiple of 16, K not a multiple of 32) and one to three levels, for the
Poisson and the Helmholtz plans: the FFT passes within 1e-5 (relative L2), the
GEMM passes within 4e-5 (each output of a GEMM pass sums n products in the FP32
accumulator, so its rounding grows like sqrt(n) where the FFT's grows like
log n: 1.7e-5 for the 511 x 511 Poisson solve); and a few FP32 time steps with
either form agree in their forces.
"""
import ctypes

import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

GRIDS = [(128, 128, 1, 4.0, -2.0, -2.0), (64, 48, 2, 2.0, -1.0, -0.75), (200, 120, 3, 4.0, -2.0, -1.2),
         (256, 256, 3, 4.0, -2.0, -2.0), (512, 512, 1, 4.0, -2.0, -2.0), (384, 128, 2, 6.0, -3.0, -1.0),
         (45, 27, 1, 3.0, -1.5, -0.9)]


def _solver(gp):
    import ibpm_b200 as ib
    from ibpm_b200 import configs, geometry
    grid = ib.Grid(*gp)
    geo = geometry.parse(configs.cylinder_geom(24, r=0.2 * gp[3] / 2))
    return grid, ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, 100.0), 0.01, "rk3", precision="fp32")


def _solve32(s, k, f):
    from ibpm_b200 import _native
    L = _native.lib()
    f = np.ascontiguousarray(f, dtype=np.float64)
    u = np.zeros_like(f)
    st = L.ibg_solve_fp32(s.handle, k, f.ctypes.data_as(ctypes.c_void_p), u.ctypes.data_as(ctypes.c_void_p))
    assert st == 0, L.ibg_last_error(s.handle)
    return u


@pytest.mark.parametrize("gp", GRIDS)
def test_gemm_passes_match_fft_passes_and_fp64(gp):
    from ibpm_b200 import _native
    L = _native.lib()
    grid, s = _solver(gp)
    rng = np.random.default_rng(sum(gp[:3]))
    f = rng.standard_normal(grid.scalar().shape)
    for k in (-1, 0):  # Poisson, Helmholtz of sub-step 0
        exact = s.poisson(f) if k < 0 else s.helmholtz(-0.5 * s.beta(0) / 100.0, f)
        assert L.ibg_set_dst_gemm(s.handle, 0) == 0
        u_fft = _solve32(s, k, f)
        assert L.ibg_set_dst_gemm(s.handle, 1) == 0
        u_gemm = _solve32(s, k, f)
        assert L.ibg_dst_gemm_status(s.handle) == 0
        assert rel_l2(u_fft, exact) < 1e-5, ("fft", k)
        assert rel_l2(u_gemm, exact) < 4e-5, ("gemm", k, rel_l2(u_gemm, exact))
        assert rel_l2(u_gemm, u_fft) < 4e-5
    s.close()


def test_fp32_steps_with_gemm_passes_match_fft_passes():
    """Four FP32 time steps of a two-domain cylinder with either form of the passes."""
    from ibpm_b200 import _native
    import ibpm_b200 as ib
    L = _native.lib()
    forces = []
    for gemm in (0, 1):
        grid, s = _solver((128, 96, 2, 4.0, -2.0, -1.5))
        assert L.ibg_set_dst_gemm(s.handle, gemm) == 0
        x = ib.State(grid, s.npoints)
        s.init()
        s.set_state(x, with_q=False)
        s.advance_resident(4)
        forces.append(s.force_history(4))
        assert L.ibg_dst_gemm_status(s.handle) == 0
        s.close()
    assert rel_l2(forces[1], forces[0]) < 4e-5
