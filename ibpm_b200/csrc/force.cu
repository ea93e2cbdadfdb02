// force.cu -- boundary-force solve on the device (FP64 throughout).
//
// Replaces CholeskySolver::computeFactorization / Minv (src/CholeskySolver.cc:89-108,
// :200-224), the CG loop of ConjugateGradientSolver::Minv
// (src/ConjugateGradientSolver.cc:35-65) and State::computeNetForce
// (src/State.cc:53-63).
#include "ibg_internal.cuh"
#include "ibg_force.cuh"

namespace ibg {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// block-wide sum for blockDim.x == 1024; result valid in every thread
__device__ double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
    s = warp_sum(s);
    return s;
}

// ---------------------------------------------------------------------------
// Cholesky factorisation M = L L^T of the upper triangle of M, column by
// column (the reference reads M(i, j) for j > i).  One CTA of 1024 threads.
// Mcol holds M(i, j) at Mcol[j*m + i].  Outputs: L row-major (Lr[r*m + k]),
// L column-major (Lc[k*m + r]) and the diagonal.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_chol_factor(int m, const double* __restrict__ Mcol, double* __restrict__ Lr,
                                                      double* __restrict__ Lc, double* __restrict__ diag,
                                                      int* __restrict__ status) {
    pdl_enter();
    extern __shared__ double sh[];
    double* rowc = sh;        // L(c, 0..c-1)
    double* red = sh + m;     // 32 partial sums
    __shared__ double dval;
    for (int c = 0; c < m; ++c) {
        for (int k = threadIdx.x; k < c; k += blockDim.x) rowc[k] = Lr[(size_t)c * m + k];
        __syncthreads();
        double part = 0.0;
        for (int k = threadIdx.x; k < c; k += blockDim.x) part += rowc[k] * rowc[k];
        const double s2 = block_sum(part, red);
        if (threadIdx.x == 0) {
            const double sum = Mcol[(size_t)c * m + c] - s2;
            if (!(sum > 0.0)) *status = 1;
            dval = sqrt(sum > 0.0 ? sum : 1.0);
            diag[c] = dval;
        }
        __syncthreads();
        const double d = dval;
        for (int r = c + 1 + threadIdx.x; r < m; r += blockDim.x) {
            double sum = Mcol[(size_t)r * m + c];  // M(c, r): upper triangle
            const double* lr = Lr + (size_t)r * m;
            for (int k = c - 1; k >= 0; --k) sum -= rowc[k] * lr[k];
            const double v = sum / d;
            Lr[(size_t)r * m + c] = v;
            Lc[(size_t)c * m + r] = v;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Forward then backward substitution with 32-row blocks (CholeskySolver::Minv,
// src/CholeskySolver.cc:200-224) on a vector held in shared memory: x holds b
// on entry and the solution on exit.  Needs blockDim.x == 1024.  Off-diagonal
// block products are spread over 32 warps; each diagonal block is solved by
// warp 0 with shuffles.
// ---------------------------------------------------------------------------
__device__ void chol_subst(int m, const double* __restrict__ Lr, const double* __restrict__ Lc,
                           const double* __restrict__ diag, double* x, double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nb = (m + 31) / 32;
    // forward: L y = b
    for (int I = 0; I < nb; ++I) {
        const int r0 = I * 32;
        const int r = r0 + lane;
        double acc = 0.0;
        if (r < m)
            for (int k = w; k < r0; k += 32) acc += Lc[(size_t)k * m + r] * x[k];
        red[w * 33 + lane] = acc;
        __syncthreads();
        if (w == 0) {
            double s = 0.0;
            for (int ww = 0; ww < 32; ++ww) s += red[ww * 33 + lane];
            double rhs = (r < m) ? x[r] - s : 0.0;
            double mine = 0.0;
            for (int c = 0; c < 32 && r0 + c < m; ++c) {
                const double xc = __shfl_sync(0xffffffffu, rhs, c) / diag[r0 + c];
                if (lane == c) mine = xc;
                if (lane > c && r < m) rhs -= Lc[(size_t)(r0 + c) * m + r] * xc;
            }
            if (r < m) x[r] = mine;
        }
        __syncthreads();
    }
    // backward: L^T x = y
    for (int I = nb - 1; I >= 0; --I) {
        const int r0 = I * 32;
        const int r = r0 + lane;
        double acc = 0.0;
        if (r < m)
            for (int k = r0 + 32 + w; k < m; k += 32) acc += Lr[(size_t)k * m + r] * x[k];
        red[w * 33 + lane] = acc;
        __syncthreads();
        if (w == 0) {
            double s = 0.0;
            for (int ww = 0; ww < 32; ++ww) s += red[ww * 33 + lane];
            double rhs = (r < m) ? x[r] - s : 0.0;
            double mine = 0.0;
            const int cmax = (m - r0) < 32 ? (m - r0) : 32;
            for (int c = cmax - 1; c >= 0; --c) {
                const double xc = __shfl_sync(0xffffffffu, rhs, c) / diag[r0 + c];
                if (lane == c) mine = xc;
                if (lane < c && r < m) rhs -= Lr[(size_t)(r0 + c) * m + r] * xc;
            }
            if (r < m) x[r] = mine;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(1024) k_chol_solve(int m, const double* __restrict__ Lr, const double* __restrict__ Lc,
                                                     const double* __restrict__ diag, const double* __restrict__ b,
                                                     double* __restrict__ x_out) {
    pdl_enter();
    extern __shared__ double sh[];
    double* x = sh;
    double* red = sh + m;
    for (int k = threadIdx.x; k < m; k += blockDim.x) x[k] = b[k];
    __syncthreads();
    chol_subst(m, Lr, Lc, diag, x, red);
    for (int k = threadIdx.x; k < m; k += blockDim.x) x_out[k] = x[k];
}

// M^-1 column j by substitution on e_j, one CTA per column; stored as row j
// of Minv (Minv[i*m + j] = (M^-1 e_j)_i, so that row i of Minv is contiguous).
__global__ void __launch_bounds__(1024) k_chol_inverse(int m, const double* __restrict__ Lr,
                                                       const double* __restrict__ Lc, const double* __restrict__ diag,
                                                       double* __restrict__ Minv) {
    pdl_enter();
    extern __shared__ double sh[];
    double* x = sh;
    double* red = sh + m;
    const int j = blockIdx.x;
    for (int k = threadIdx.x; k < m; k += blockDim.x) x[k] = (k == j) ? 1.0 : 0.0;
    __syncthreads();
    chol_subst(m, Lr, Lc, diag, x, red);
    for (int k = threadIdx.x; k < m; k += blockDim.x) Minv[(size_t)k * m + j] = x[k];
}

// y = Minv b: one warp per row
__global__ void k_minv_apply(int m, const double* __restrict__ Minv, const double* __restrict__ b,
                             double* __restrict__ y) {
    pdl_enter();
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= m) return;
    const double* a = Minv + (size_t)row * m;
    double acc = 0.0;
    for (int k = lane; k < m; k += 32) acc += a[k] * b[k];
    acc = warp_sum(acc);
    if (lane == 0) y[row] = acc;
}

// ---------------------------------------------------------------------------
// CG (absolute tolerance on r.r, warm start from x), one CTA per update.
// scal: [0] delta, [1] delta_old, [2] tol^2 ; flags: [0] active, [1] iterations, [2] max iterations
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_cg_begin(int m, const double* __restrict__ b, const double* __restrict__ Mx,
                                                   double* __restrict__ r, double* __restrict__ d,
                                                   double* __restrict__ scal, int* __restrict__ flags) {
    pdl_enter();
    __shared__ double red[32];
    double part = 0.0;
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        const double rv = b[k] - Mx[k];
        r[k] = rv;
        d[k] = rv;
        part += rv * rv;
    }
    const double delta = block_sum(part, red);
    if (threadIdx.x == 0) {
        scal[0] = delta;
        flags[1] = 0;
        flags[0] = (delta > scal[2] && flags[2] > 0) ? 1 : 0;
    }
}

__global__ void __launch_bounds__(1024) k_cg_update(int m, double* __restrict__ x, double* __restrict__ r,
                                                    double* __restrict__ d, const double* __restrict__ q,
                                                    double* __restrict__ scal, int* __restrict__ flags) {
    pdl_enter();
    __shared__ double red[32];
    if (flags[0] == 0) return;
    double part = 0.0;
    for (int k = threadIdx.x; k < m; k += blockDim.x) part += d[k] * q[k];
    const double dq = block_sum(part, red);
    const double delta = scal[0];
    const double alpha = delta / dq;
    part = 0.0;
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        x[k] = x[k] + alpha * d[k];
        const double rv = r[k] - alpha * q[k];
        r[k] = rv;
        part += rv * rv;
    }
    const double dn = block_sum(part, red);
    const double beta = dn / delta;
    for (int k = threadIdx.x; k < m; k += blockDim.x) d[k] = r[k] + beta * d[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        scal[1] = delta;
        scal[0] = dn;
        const int it = flags[1] + 1;
        flags[1] = it;
        flags[0] = (dn > scal[2] && it < flags[2]) ? 1 : 0;
        if (!(dn == dn)) flags[0] = 0;  // NaN stops the loop
    }
}

// ---------------------------------------------------------------------------
// flexible preconditioned CG (one CTA per update).  scal: [0] r.z, [2] tol^2,
// [3] r.r; flags: [0] active, [1] iterations, [2] max iterations
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_pcg_begin(int m, const double* __restrict__ b, const double* __restrict__ Mx,
                                                    double* __restrict__ r, double* __restrict__ scal,
                                                    int* __restrict__ flags) {
    pdl_enter();
    __shared__ double red[32];
    double part = 0.0;
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        const double rv = b[k] - Mx[k];
        r[k] = rv;
        part += rv * rv;
    }
    const double rr = block_sum(part, red);
    if (threadIdx.x == 0) {
        scal[3] = rr;
        flags[1] = 0;
        flags[8] = 0;  // preconditioner in use (no fallback yet)
    }
}

__global__ void __launch_bounds__(1024) k_pcg_begin2(int m, const double* __restrict__ r, double* __restrict__ z,
                                                     double* __restrict__ d, double* __restrict__ scal,
                                                     int* __restrict__ flags) {
    pdl_enter();
    __shared__ double red[32];
    double part = 0.0;
    for (int k = threadIdx.x; k < m; k += blockDim.x) part += r[k] * z[k];
    const double rz = block_sum(part, red);
    // a preconditioner that is not positive on the first residual: plain CG from the start
    const bool fallback = !(rz > 0.0);
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        const double v = fallback ? r[k] : z[k];
        z[k] = v;
        d[k] = v;
    }
    if (threadIdx.x == 0) {
        const double rr = scal[3];
        scal[0] = fallback ? rr : rz;
        flags[8] = fallback ? 1 : 0;
        flags[0] = (rr > scal[2] && flags[2] > 0 && rr == rr) ? 1 : 0;
    }
}

__global__ void __launch_bounds__(1024) k_pcg_step1(int m, double* __restrict__ x, double* __restrict__ r,
                                                    const double* __restrict__ d, const double* __restrict__ q,
                                                    const double* __restrict__ z, double* __restrict__ zold,
                                                    double* __restrict__ scal, int* __restrict__ flags) {
    pdl_enter();
    __shared__ double red[32];
    if (flags[0] == 0) return;
    double part = 0.0;
    for (int k = threadIdx.x; k < m; k += blockDim.x) part += d[k] * q[k];
    const double dq = block_sum(part, red);
    const double alpha = scal[0] / dq;
    part = 0.0;
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        x[k] = x[k] + alpha * d[k];
        const double rv = r[k] - alpha * q[k];
        r[k] = rv;
        zold[k] = z[k];
        part += rv * rv;
    }
    const double rr = block_sum(part, red);
    if (threadIdx.x == 0) scal[3] = rr;
}

__global__ void __launch_bounds__(1024) k_pcg_step2(int m, const double* __restrict__ r, double* __restrict__ z,
                                                    const double* __restrict__ zold, double* __restrict__ d,
                                                    double* __restrict__ scal, int* __restrict__ flags) {
    pdl_enter();
    __shared__ double red[32];
    __shared__ int restart;
    if (flags[0] == 0) return;
    double p1 = 0.0, p2 = 0.0, p3 = 0.0;
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        p1 += r[k] * z[k];
        p2 += r[k] * zold[k];
        p3 += r[k] * r[k];
    }
    const double rz = block_sum(p1, red);
    const double rzo = block_sum(p2, red);
    const double rr = block_sum(p3, red);
    const int it = flags[1] + 1;
    if (threadIdx.x == 0) {
        // fall back to plain CG (restart with d = r) when the preconditioner is not
        // positive on r or has not converged within its iteration budget
        restart = (flags[8] == 0 && (!(rz > 0.0) || it >= flags[9])) ? 1 : 0;
    }
    __syncthreads();
    if (restart) {
        for (int k = threadIdx.x; k < m; k += blockDim.x) {
            z[k] = r[k];
            d[k] = r[k];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            flags[8] = 1;
            scal[0] = rr;
            flags[1] = it;
            flags[0] = (rr > scal[2] && it < flags[2] && rr == rr) ? 1 : 0;
        }
        return;
    }
    const double beta = (rz - rzo) / scal[0];  // Polak-Ribiere
    for (int k = threadIdx.x; k < m; k += blockDim.x) d[k] = z[k] + beta * d[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        scal[0] = rz;
        flags[1] = it;
        flags[0] = (rr > scal[2] && it < flags[2] && rz > 0.0 && rr == rr) ? 1 : 0;
    }
}

// net force sum(f) dx^2 in each direction, appended to a history buffer
__global__ void k_net_force(int npts, const double* __restrict__ f, double dx2, double* __restrict__ out) {
    pdl_enter();
    double sx = 0.0, sy = 0.0;
    for (int k = threadIdx.x; k < npts; k += 32) {
        sx += f[k];
        sy += f[npts + k];
    }
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    if (threadIdx.x == 0) {
        out[0] = sx * dx2;
        out[1] = sy * dx2;
    }
}

__global__ void k_add_time(double* t, double dt) {
    pdl_enter();
    if (threadIdx.x == 0 && blockIdx.x == 0) *t = *t + dt;
}

// ---------------------------------------------------------------------------
int chol_factor(int m, const double* Mcol, double* Lr, double* Lc, double* diag, int* d_status, cudaStream_t st) {
    const size_t sm = sizeof(double) * (m + 32);
    if (sm > 200 * 1024) return IBG_ERR_UNSUPPORTED;
    if (raise_smem_limit((const void*)k_chol_factor, (int)sm)) return IBG_ERR_CUDA;
    cudaMemsetAsync(d_status, 0, sizeof(int), st);
    cudaMemsetAsync(Lr, 0, sizeof(double) * m * m, st);
    cudaMemsetAsync(Lc, 0, sizeof(double) * m * m, st);
    launch_k(k_chol_factor, 1, 1024, sm, st, m, Mcol, Lr, Lc, diag, d_status);
    return cudaPeekAtLastError() == cudaSuccess ? IBG_OK : IBG_ERR_CUDA;
}

void chol_solve(int m, const double* Lr, const double* Lc, const double* diag, const double* b, double* x,
                cudaStream_t st) {
    const size_t sm = sizeof(double) * (m + 32 * 33);
    launch_k(k_chol_solve, 1, 1024, sm, st, m, Lr, Lc, diag, b, x);
}

int chol_solve_prepare(int m) {
    const size_t sm = sizeof(double) * (m + 32 * 33);
    if (sm > 200 * 1024) return IBG_ERR_UNSUPPORTED;
    if (raise_smem_limit((const void*)k_chol_solve, (int)sm) || raise_smem_limit((const void*)k_chol_inverse, (int)sm))
        return IBG_ERR_CUDA;
    return IBG_OK;
}

void chol_inverse(int m, const double* Lr, const double* Lc, const double* diag, double* Minv, cudaStream_t st) {
    const size_t sm = sizeof(double) * (m + 32 * 33);
    launch_k(k_chol_inverse, m, 1024, sm, st, m, Lr, Lc, diag, Minv);
}

void minv_apply(int m, const double* Minv, const double* b, double* y, cudaStream_t st) {
    launch_k(k_minv_apply, (m + 7) / 8, 256, 0, st, m, Minv, b, y);
}

void cg_begin(int m, const double* b, const double* Mx, double* r, double* d, double* scal, int* flags,
              cudaStream_t st) {
    launch_k(k_cg_begin, 1, 1024, 0, st, m, b, Mx, r, d, scal, flags);
}

void cg_update(int m, double* x, double* r, double* d, const double* q, double* scal, int* flags, cudaStream_t st) {
    launch_k(k_cg_update, 1, 1024, 0, st, m, x, r, d, q, scal, flags);
}

void pcg_begin(int m, const double* b, const double* Mx, double* r, double* scal, int* flags, cudaStream_t st) {
    launch_k(k_pcg_begin, 1, 1024, 0, st, m, b, Mx, r, scal, flags);
}
void pcg_begin2(int m, const double* r, double* z, double* d, double* scal, int* flags, cudaStream_t st) {
    launch_k(k_pcg_begin2, 1, 1024, 0, st, m, r, z, d, scal, flags);
}
void pcg_step1(int m, double* x, double* r, const double* d, const double* q, const double* z, double* zold,
               double* scal, int* flags, cudaStream_t st) {
    launch_k(k_pcg_step1, 1, 1024, 0, st, m, x, r, d, q, z, zold, scal, flags);
}
void pcg_step2(int m, const double* r, double* z, const double* zold, double* d, double* scal, int* flags,
               cudaStream_t st) {
    launch_k(k_pcg_step2, 1, 1024, 0, st, m, r, z, zold, d, scal, flags);
}

void net_force(int npts, const double* f, double dx2, double* out, cudaStream_t st) {
    launch_k(k_net_force, 1, 32, 0, st, npts, f, dx2, out);
}

void add_time(double* t, double dt, cudaStream_t st) { launch_k(k_add_time, 1, 32, 0, st, t, dt); }

}  // namespace ibg
