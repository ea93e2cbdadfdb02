"""The FP32 plans' eigenvalue tables, checked on the CPU.

The reference's Laplacian eigenvalues are lambda_kl = 2 (cos(pi k / nx) + cos(pi l / ny) - 2) / dx^2
(src/EllipticSolver2d.cc:42-54).  For the lowest modes the sum cancels to about (pi / n)^2, so formed
from FP32 cosines (absolute error ~6e-8) it loses about three digits at n = 512.  The FP32 tables
(ibpm_b200/csrc/elliptic.cu, the grid tables' set-up) hold cos(theta) - 1 = -2 sin^2(theta / 2),
tabulated in double and rounded once, and the FP32 kernels form lambda = 2 (cx + cy) / dx^2
(eig_inverse in ibg_kernels.cuh).  This test emulates both in float32 and holds the kernels' form to
a few float32 roundings over every mode, against the reference's formula in float64.
"""
import numpy as np
import pytest


def _reference(nx, ny, dx):
    k = np.arange(1, nx)[:, None]
    l = np.arange(1, ny)[None, :]
    return 2.0 * (np.cos(np.pi * k / nx) + np.cos(np.pi * l / ny) - 2.0) / (dx * dx)


def _fp32_cosines(nx, ny, dx):
    cx = np.cos(np.pi * np.arange(1, nx) / nx).astype(np.float32)[:, None]
    cy = np.cos(np.pi * np.arange(1, ny) / ny).astype(np.float32)[None, :]
    return np.float32(2) * (cx + cy - np.float32(2)) * np.float32(1.0 / (dx * dx))


def _fp32_cos_minus_one(nx, ny, dx):
    cx = (-2.0 * np.sin(np.pi * np.arange(1, nx) / (2 * nx)) ** 2).astype(np.float32)[:, None]
    cy = (-2.0 * np.sin(np.pi * np.arange(1, ny) / (2 * ny)) ** 2).astype(np.float32)[None, :]
    return np.float32(2) * (cx + cy) * np.float32(1.0 / (dx * dx))


@pytest.mark.parametrize("nx,ny", [(128, 128), (256, 256), (512, 512), (1024, 1024), (400, 200)])
def test_fp32_eigenvalues_keep_their_digits(nx, ny):
    dx = 4.0 / nx
    ref = _reference(nx, ny, dx)
    rel_kernel = np.abs(_fp32_cos_minus_one(nx, ny, dx).astype(np.float64) - ref) / np.abs(ref)
    rel_naive = np.abs(_fp32_cosines(nx, ny, dx).astype(np.float64) - ref) / np.abs(ref)
    eps32 = float(np.finfo(np.float32).eps)
    assert rel_kernel.max() <= 4 * eps32  # a few roundings, whatever the mode
    if nx >= 256:
        # the cosine form loses digits on the lowest mode (what the tables avoid)
        assert rel_naive[0, 0] > 100 * eps32
