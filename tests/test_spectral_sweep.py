"""The multi-domain solve as the kernels organise it, restated in numpy and checked on the CPU.

The reference solves the levels one after another, coarse to fine, each level a 2-D DST-I solve whose
Dirichlet values come from the coarser level's solution (src/EllipticSolver.cc:47-73,
src/EllipticSolver2d.cc:87-95, getBC src/Scalar.cc:91-127).  The kernels (ibpm_b200/csrc/elliptic.cu)
move that coupling into the transform domain so that every level's forward and inverse transforms run
in one launch each:

1. coarsify the right-hand side (k_coarsify), forward rows and columns of every level (k_dst_rows,
   k_dst_cols): F_l;
2. coarse to fine: U_l = E_l (F_l - c_l Slift_l), where Slift_l = sy1 B + syn T + sx1 L + sxn R holds
   the 1-D DSTs B, T, L, R of level l's boundary values (lifted_coef).  Those boundary values are the
   coarser level's solution on four of its lines: on row line j0 the solution is norm * DST(U s_j0),
   s_j0[l] = 2 sin(pi (l + 1) j0 / ny) -- a row sum of U (k_sweep_sums) followed by a line DST, getBC's
   copy/average interpolation and the boundary DST (the lines step, or the edge map that does it as
   one matrix: A = D P norm D, the same for both lines of a direction and for every level);
3. inverse columns and rows of every level with U_l (k_dst_cols mode 3, k_dst_rows).

These tests hold that restatement to the oracle's level-by-level solve (itself pinned to the
reference), and check the edge-map form of the lines step; they need no GPU.
"""
import numpy as np
import pytest

from oracle import ibpm_oracle as O


def _sines(n, pos):
    """2 sin(pi (k + 1) pos / n), k = 0 .. n - 2: the DST-I basis evaluated at node `pos`."""
    return 2.0 * np.sin(np.pi * np.arange(1, n) * pos / n)


def _interp(line, n, ext):
    """getBC along one boundary of the finer level: coarse line values (nodes 1 .. n-1) -> the n + 1
    fine boundary values (coincident nodes copied, the others averaged)."""
    padded = np.concatenate([[0.0], line, [0.0]])
    i = np.arange(n + 1)
    ii = i // 2 + ext
    a, b = padded[ii], padded[np.minimum(ii + 1, n)]
    return np.where(i % 2 == 1, 0.5 * (a + b), a)


def lines_step(V, n, ext, norm):
    """One direction's lines step: the sums V (one row sum per coarse line) -> the finer level's
    boundary DST along that direction."""
    vals = norm * O.dst1(V, -1)                # the coarser level's solution on the line
    bnd = _interp(vals, n, ext)                 # the finer level's boundary values (0 .. n)
    return O.dst1(bnd[1:n], -1)                 # their DST over the interior nodes


def edge_map(n, ext, norm):
    """The lines step as a matrix (k_edge_map applies the step to unit vectors)."""
    return np.stack([lines_step(e, n, ext, norm) for e in np.eye(n - 1)], axis=1)


def spectral_solve(g, kind, f, alpha=0.0, use_edge_maps=False):
    nx, ny, L = g.nx, g.ny, g.ngrid
    nxe, nye = g.nxext, g.nyext
    rhs = O.coarsify(g, f)
    F = [O.dst1(O.dst1(rhs[l], -2), -1) for l in range(L)]
    norm = 1.0 / (2 * nx * 2 * ny)
    sy1, syn = _sines(ny, 1), _sines(ny, ny - 1)
    sx1, sxn = _sines(nx, 1), _sines(nx, nx - 1)
    Ax, Ay = (edge_map(nx, nxe, norm), edge_map(ny, nye, norm)) if use_edge_maps else (None, None)
    U = [None] * L
    for lev in range(L - 1, -1, -1):
        E = O.eigen_inverse(kind, nx, ny, g.dx_lev(lev), alpha)
        R = F[lev]
        if lev < L - 1:
            Uc = U[lev + 1]
            # row sums on the coarser level's lines j0 = nye (bottom) and ny/2 + nye (top), column sums
            # on i0 = nxe (left) and nx/2 + nxe (right)
            Vb, Vt = Uc @ _sines(ny, nye), Uc @ _sines(ny, ny // 2 + nye)
            Wl, Wr = Uc.T @ _sines(nx, nxe), Uc.T @ _sines(nx, nx // 2 + nxe)
            if use_edge_maps:
                B, T, Lf, Rt = Ax @ Vb, Ax @ Vt, Ay @ Wl, Ay @ Wr
            else:
                B, T = lines_step(Vb, nx, nxe, norm), lines_step(Vt, nx, nxe, norm)
                Lf, Rt = lines_step(Wl, ny, nye, norm), lines_step(Wr, ny, nye, norm)
            slift = np.outer(B, sy1) + np.outer(T, syn) + np.outer(sx1, Lf) + np.outer(sxn, Rt)
            dx = g.dx_lev(lev)
            c = (1.0 / (dx * dx)) if kind == "poisson" else (alpha / (dx * dx))
            R = R - c * slift
        U[lev] = E * R
    return np.stack([norm * O.dst1(O.dst1(U[l], -2), -1) for l in range(L)])


GRIDS = [(32, 32, 3, 2.0), (40, 24, 2, 3.0), (36, 22, 3, 2.0), (48, 64, 4, 4.0), (28, 28, 1, 1.0)]


@pytest.mark.parametrize("edge_maps", [False, True], ids=["lines", "edge_maps"])
@pytest.mark.parametrize("kind,alpha", [("poisson", 0.0), ("helmholtz", -0.0125)])
@pytest.mark.parametrize("gp", GRIDS)
def test_spectral_sweep_matches_level_by_level_solve(gp, kind, alpha, edge_maps):
    nx, ny, ngrid, length = gp
    g = O.Grid(nx, ny, ngrid, length, -length / 2, -length / 2)
    rng = np.random.default_rng(nx * 1000 + ny * 10 + ngrid)
    f = rng.standard_normal(g.scalar().shape)
    ref = O.EllipticSolver(g, kind, alpha).solve(f)
    got = spectral_solve(g, kind, f, alpha, use_edge_maps=edge_maps)
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)


def test_edge_map_is_shared_by_the_lines_of_a_direction():
    """The map from a line's sums to the finer level's boundary DST depends on neither the line's
    position (that enters through the sine vector of the sums) nor the level: one matrix per direction."""
    nx, nxe = 40, 10
    norm = 1.0 / (4 * nx * 24)
    A = edge_map(nx, nxe, norm)
    rng = np.random.default_rng(3)
    for _ in range(3):
        V = rng.standard_normal(nx - 1)
        assert np.allclose(A @ V, lines_step(V, nx, nxe, norm), rtol=0, atol=1e-13 * np.abs(V).sum())
