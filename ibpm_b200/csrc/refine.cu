// refine.cu -- one step of iterative refinement for the multi-domain solves of
// the FP32-transform form (IBG_PRECISION_FP32_REFINED).
//
// The reference solves every level of a multi-domain Poisson or Helmholtz
// problem in FP64 (src/EllipticSolver.cc:47-73, src/EllipticSolver2d.cc:53-110).
// Here a solve with an FP64 right-hand side f and an FP64 result u runs as
//   u1 = S32(f)              FP32 transforms (f rounded to FP32 after coarsify)
//   r  = f - A u1            residual of every level in FP64, with each level's
//                            boundary values taken from the coarser level's u1
//                            (Scalar::getBC, src/Scalar.cc:91-127), zero on the
//                            coarsest; A = L (Poisson) or 1 + alpha L (Helmholtz),
//                            L the 5-point Laplacian whose Dirichlet eigenvalues
//                            2 (cos(pi i/nx) + cos(pi j/ny) - 2) / dx^2 the DST
//                            solve divides by (src/EllipticSolver2d.cc:42-54)
//   d  = S32(r)              the same FP32 solve, level by level, without
//                            coarsifying r again (r is already per level)
//   u  = u1 + d              accumulated in FP64
// Every level's problem is linear in its right-hand side and its boundary
// values, so u + d solves the coupled levels exactly up to the FP32 error of d,
// which is the FP32 error of u1 times the FP32 relative error of a solve.
#include "ibg_internal.cuh"
#include "ibg_kernels.cuh"

namespace ibg {

namespace {

__device__ __forceinline__ bool in_overlap(const GridDev& g, int i, int j) {
    return i > g.nxe && i < g.nx / 2 + g.nxe && j > g.nye && j < g.ny / 2 + g.nye;
}

// node (i, j) of level values `u` (FP32) as FP64, 0 <= i <= nx, 0 <= j <= ny: the
// boundary ring from the coarser level `c` (copy at coincident nodes, the FP64
// mean of the two neighbours in between), zero when c == nullptr
__device__ __forceinline__ double node_bc64(const float* u, const float* c, const GridDev& g, int i, int j) {
    if (i >= 1 && i <= g.nx - 1 && j >= 1 && j <= g.ny - 1) return (double)node(u, g, i, j);
    if (c == nullptr) return 0.0;
    int ii, jj, di = 0, dj = 0;
    bool odd;
    if (j == 0 || j == g.ny) {
        ii = i / 2 + g.nxe;
        jj = (j == 0) ? g.nye : g.ny / 2 + g.nye;
        odd = (i & 1) != 0;
        di = 1;
    } else {
        ii = (i == 0) ? g.nxe : g.nx / 2 + g.nxe;
        jj = j / 2 + g.nye;
        odd = (j & 1) != 0;
        dj = 1;
    }
    const double a = (double)node(c, g, ii, jj);
    if (!odd) return a;
    return 0.5 * (a + (double)node(c, g, ii + di, jj + dj));
}

}  // namespace

// out = (float)(s * rhs): every level of f, with the overlap interiors of levels
// >= 1 taken from the coarsified values rc
__global__ void k_refine_prep(GridDev g, const double* __restrict__ f, const double* __restrict__ rc, double s,
                              float* __restrict__ out) {
    pdl_enter();
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.N1) return;
    const int lev = blockIdx.y;
    const size_t k = (size_t)lev * g.N1 + n;
    const int i = n / g.NJ + 1, j = n % g.NJ + 1;
    const double v = (lev >= 1 && in_overlap(g, i, j)) ? rc[k] : f[k];
    out[k] = (float)(s * v);
}

// r = s * rhs - A u of every level in FP64, stored as FP32
template <bool HELM>
__global__ void k_refine_residual(GridDev g, const double* __restrict__ f, const double* __restrict__ rc, double s,
                                  const float* __restrict__ u, double alpha, float* __restrict__ r) {
    pdl_enter();
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.N1) return;
    const int lev = blockIdx.y;
    const size_t k = (size_t)lev * g.N1 + n;
    const int i = n / g.NJ + 1, j = n % g.NJ + 1;
    const float* ul = u + (size_t)lev * g.N1;
    const float* uc = (lev + 1 < g.L) ? u + (size_t)(lev + 1) * g.N1 : nullptr;
    const double dxl = lev_dx(g, lev);
    const double c = (double)ul[n];
    const double lap = (node_bc64(ul, uc, g, i + 1, j) + node_bc64(ul, uc, g, i - 1, j) +
                        node_bc64(ul, uc, g, i, j + 1) + node_bc64(ul, uc, g, i, j - 1) - 4.0 * c) /
                       (dxl * dxl);
    const double Au = HELM ? c + alpha * lap : lap;
    const double rhs = s * ((lev >= 1 && in_overlap(g, i, j)) ? rc[k] : f[k]);
    r[k] = (float)(rhs - Au);
}

// u = u1 + d in FP64; optionally out2 = base - u
__global__ void k_refine_finish(size_t n, const float* __restrict__ u1, const float* __restrict__ d,
                                double* __restrict__ u, double* __restrict__ out2, const double* __restrict__ base) {
    pdl_enter();
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double v = (double)u1[k] + (double)d[k];
    u[k] = v;
    if (out2) out2[k] = base[k] - v;
}

int refined_solve(const GridDev& g, const EllipticPlan<float>& plan32, const SolveCall<double>& c, double* rc64,
                  float* f32, float* u32, float* d32, float* tbuf32, float* tbuf2_32, float* sweep32, cudaStream_t st) {
    if (c.batch != 1) return IBG_ERR_ARG;
    const size_t S = (size_t)g.L * g.N1;
    const dim3 grid((unsigned)((g.N1 + 255) / 256), (unsigned)g.L);
    if (g.L > 1) coarsify_rhs(g, c.f, rc64, st);
    launch_k(k_refine_prep, grid, 256, 0, st, g, c.f, (const double*)rc64, (double)c.in_scale, f32);
    SolveCall<float> s{};
    s.f = f32;
    s.u = u32;
    s.rc = nullptr;  // the right-hand side is coarsified already
    s.tbuf = tbuf32;
    s.tbuf2 = tbuf2_32;
    s.sweep = sweep32;
    s.bstride = S;
    s.batch = 1;
    s.in_scale = 1.0f;
    int e = plan32.solve(s, st);
    if (e) return e;
    if (plan32.helmholtz)
        launch_k(k_refine_residual<true>, grid, 256, 0, st, g, c.f, (const double*)rc64, (double)c.in_scale,
                 (const float*)u32, plan32.alpha, f32);
    else
        launch_k(k_refine_residual<false>, grid, 256, 0, st, g, c.f, (const double*)rc64, (double)c.in_scale,
                 (const float*)u32, 0.0, f32);
    s.u = d32;
    e = plan32.solve(s, st);
    if (e) return e;
    launch_k(k_refine_finish, (unsigned)((S + 255) / 256), 256, 0, st, S, (const float*)u32, (const float*)d32, c.u,
             c.out2, c.base);
    return cudaPeekAtLastError() == cudaSuccess ? IBG_OK : IBG_ERR_CUDA;
}

int refined_solve_launches(const GridDev& g, const EllipticPlan<float>& plan32) {
    return (g.L - 1) + 1 + 2 * plan32.launches(false) + 2;
}

}  // namespace ibg
