"""The FP32-transform solve with one FP64-residual refinement, emulated in numpy on the CPU.

ibpm_b200/csrc/refine.cu runs a multi-domain Poisson or Helmholtz solve (the reference's
src/EllipticSolver.cc:47-73 in FP64) as: u1 = S32(f) with FP32 transforms; r = f - A u1 for every
level in FP64, each level's boundary values taken from the coarser level's u1 (getBC,
src/Scalar.cc:91-127), stored in FP32; d = S32(r) without coarsifying again; u = u1 + d in FP64.
Every level's problem is linear in its right-hand side and its boundary values, so the correction
removes u1's error up to the FP32 error of d.  This test emulates S32 in float32 (float32 DSTs,
eigen-inverse from the cos - 1 tables, lifting and interpolation in float32) and checks that one
refinement takes the error against the oracle's FP64 solve from the FP32 level (~1e-7) to below
1e-12, on several grids, Poisson and Helmholtz (alpha < 0, as the time step's 1 - (dt / 2 Re) L).
"""
import numpy as np
import pytest

from oracle import ibpm_oracle as O


def _dst1_32(x, axis):
    x = np.moveaxis(x.astype(np.float32), axis, -1)
    n = x.shape[-1]
    ext = np.zeros(x.shape[:-1] + (2 * (n + 1),), np.float32)
    ext[..., 1:n + 1] = x
    ext[..., n + 2:] = -x[..., ::-1]
    y = (-np.fft.fft(ext, axis=-1)[..., 1:n + 1].imag).astype(np.float32)
    return np.moveaxis(y, -1, axis)


def _eig_inverse32(kind, nx, ny, dx, alpha):
    cx = (-2.0 * np.sin(np.pi * np.arange(1, nx) / (2 * nx)) ** 2).astype(np.float32)[:, None]
    cy = (-2.0 * np.sin(np.pi * np.arange(1, ny) / (2 * ny)) ** 2).astype(np.float32)[None, :]
    lam = np.float32(2) * (cx + cy) * np.float32(1.0 / (dx * dx))
    if kind == "poisson":
        return np.float32(1) / lam
    return np.float32(1) / (np.float32(1) + np.float32(alpha) * lam)


def _solve_levels32(g, kind, alpha, rhs32):
    """S32 on a right-hand side that is already per level (coarsified): coarse to fine, FP32."""
    nx, ny = g.nx, g.ny
    u = np.zeros_like(rhs32, dtype=np.float32)
    norm = np.float32(1.0 / (2 * nx * 2 * ny))
    for lev in range(g.ngrid - 1, -1, -1):
        r = rhs32[lev].copy()
        if lev < g.ngrid - 1:
            dx = g.dx_lev(lev)
            c = np.float32((1.0 / (dx * dx)) if kind == "poisson" else (alpha / (dx * dx)))
            r = O.lift_bc(r, O.get_bc(g, u, lev), c).astype(np.float32)
        E = _eig_inverse32(kind, nx, ny, g.dx_lev(lev), alpha)
        u[lev] = _dst1_32(_dst1_32(_dst1_32(_dst1_32(r, -2), -1) * E, -2), -1) * norm
    return u


def _residual64(g, kind, alpha, rhs, u32):
    """rhs - A u1 of every level in FP64, boundary ring from the coarser level's u1 (zero outermost)."""
    u = u32.astype(np.float64)
    r = np.empty_like(rhs)
    for lev in range(g.ngrid):
        bc = O.get_bc(g, u, lev) if lev < g.ngrid - 1 else O.zero_bc(g)
        p = O._with_bc(g, u, lev, bc)
        dx = g.dx_lev(lev)
        lap = (p[2:, 1:-1] + p[:-2, 1:-1] + p[1:-1, 2:] + p[1:-1, :-2] - 4.0 * p[1:-1, 1:-1]) / (dx * dx)
        Au = lap if kind == "poisson" else u[lev] + alpha * lap
        r[lev] = rhs[lev] - Au
    return r


@pytest.mark.parametrize("kind,alpha", [("poisson", 0.0), ("helmholtz", -0.0125)])
@pytest.mark.parametrize("gp", [(64, 64, 3, 2.0), (80, 40, 2, 4.0), (96, 96, 4, 4.0), (128, 128, 1, 2.0)])
def test_one_refinement_reaches_fp64_accuracy(gp, kind, alpha):
    nx, ny, ngrid, length = gp
    g = O.Grid(nx, ny, ngrid, length, -length / 2, -length / 2)
    rng = np.random.default_rng(nx + ny + ngrid)
    f = rng.standard_normal(g.scalar().shape)
    ref = O.EllipticSolver(g, kind, alpha).solve(f)
    rhs = O.coarsify(g, f)
    u1 = _solve_levels32(g, kind, alpha, rhs.astype(np.float32))
    r = _residual64(g, kind, alpha, rhs, u1).astype(np.float32)
    d = _solve_levels32(g, kind, alpha, r)
    u = u1.astype(np.float64) + d.astype(np.float64)
    e1 = np.linalg.norm(u1 - ref) / np.linalg.norm(ref)
    e2 = np.linalg.norm(u - ref) / np.linalg.norm(ref)
    assert 1e-9 < e1 < 1e-5  # the FP32 solve alone
    assert e2 < 1e-12        # after one FP64-residual refinement (7e-15 .. 8e-14 measured)
