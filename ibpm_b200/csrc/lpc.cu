// lpc.cu -- learned preconditioner for the moving-body force solve.
//
// The reference solves M f = r, M = C A^-1 B, by plain CG whenever the bodies
// move (src/ConjugateGradientSolver.cc:35-65), because M changes every step.
// Here a network maps the current body geometry to an approximate inverse K of
// M, used as the preconditioner of the flexible CG (z = K r: linear in the
// residual, so the usual PCG theory applies).
//
// Per boundary point i: g_i = (x, y, nx, ny) (position about its body's
// centroid over the body's extent, unit normal), gbar_i = mean of g_j over its
// up to 8 boundary neighbours (i +- 1..4 along the body).  For every ordered
// pair (i, j):
//   x_ij = [g_i, gbar_i, g_j, gbar_j, x_i - x_j, y_i - y_j, |p_i - p_j|]     19
//   h1   = relu(W1 x_ij + b1)                                          19 -> 256
//   h2   = relu(W2 h1 + b2)                                           256 -> 256
//   k_ij = W3 h2 + b3                                                 256 -> 4
// k_ij is the 2 x 2 block coupling force component c at j to component a at i:
// Kraw[a P + i][c P + j] = k_ij[2a + c]; K = (Kraw + Kraw^T) / 2, and the
// preconditioner of sub-step k is K / (c0 beta_k), c0 the mean diagonal of
// M / beta over the training configurations (stored after the weights).
//
// Training data are what the solver generates with its exact operator: the
// columns of M = beta C A^-1 B at sampled body configurations, i.e. the pairs
// (residual M e_j, exact force e_j).  Loss (FP32): mean over configurations of
// |K Mn - I|_F^2 / m with Mn = M / (beta c0), minimised by Adam with the
// hand-written backward pass below.  Inference runs with BF16 weights and
// activations (FP32 accumulation) and writes K in FP64.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/ibpm_b200.h"
#include "ibg_internal.cuh"
#include "ibg_lpc.cuh"

namespace ibg {

// parameter layout (floats)
constexpr int kF = 19, kH = 256, kO = 4;
constexpr size_t oW1 = 0, oB1 = oW1 + (size_t)kH * kF, oW2 = oB1 + kH, oB2 = oW2 + (size_t)kH * kH,
                 oW3 = oB2 + kH, oB3 = oW3 + (size_t)kO * kH, oC0 = oB3 + kO, kNParams = oC0 + 1;

size_t lpc_num_params() { return kNParams; }

// ---------------------------------------------------------------------------
// generic batched FP32 GEMM: C[z][M x N] = alpha op(A) op(B) + beta C, element
// (i, k) of op(A) at A[z sA + i as0 + k as1], (k, j) of op(B) at
// B[z sB + k bs0 + j bs1].  64 x 64 tiles, 256 threads, 4 x 4 outputs per thread.
// With kchunk > 0, item z covers K indices [z kchunk, min(K, (z + 1) kchunk)) (split-K:
// sA, sB step over K and C[z] receives the partial product).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, float alpha, const float* __restrict__ A,
                                               long as0, long as1, long sA, const float* __restrict__ B, long bs0,
                                               long bs1, long sB, float beta, float* __restrict__ C, long ldc,
                                               long sC, long kchunk) {
    __shared__ float As[16][64 + 1];
    __shared__ float Bs[16][64 + 1];
    A += blockIdx.z * sA;
    B += blockIdx.z * sB;
    C += blockIdx.z * sC;
    if (kchunk > 0) {
        const long rest = (long)K - (long)blockIdx.z * kchunk;
        K = (int)(rest < kchunk ? rest : kchunk);
    }
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const long i0 = (long)blockIdx.y * 64, j0 = (long)blockIdx.x * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int t = threadIdx.x; t < 16 * 64; t += 256) {
            // consecutive threads walk the operand's contiguous index
            int kk, ii;
            if (as1 == 1) { kk = t % 16; ii = t / 16; } else { kk = t / 64; ii = t % 64; }
            const long gi = i0 + ii;
            const int gk = k0 + kk;
            As[kk][ii] = (gi < M && gk < K) ? A[gi * as0 + gk * as1] : 0.f;
            int kb, jj;
            if (bs0 == 1) { kb = t % 16; jj = t / 16; } else { kb = t / 64; jj = t % 64; }
            const long gj = j0 + jj;
            const int gkb = k0 + kb;
            Bs[kb][jj] = (gkb < K && gj < N) ? B[gkb * bs0 + gj * bs1] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) a[r] = As[kk][ty * 4 + r];
#pragma unroll
            for (int c = 0; c < 4; ++c) b[c] = Bs[kk][tx * 4 + c];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] += a[r] * b[c];
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const long gi = i0 + ty * 4 + r;
        if (gi >= M) continue;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const long gj = j0 + tx * 4 + c;
            if (gj >= N) continue;
            float v = alpha * acc[r][c];
            if (beta != 0.f) v += beta * C[gi * ldc + gj];
            C[gi * ldc + gj] = v;
        }
    }
}

static void sgemm(long M, int N, int K, float alpha, const float* A, long as0, long as1, const float* B, long bs0,
                  long bs1, float beta, float* C, long ldc, cudaStream_t st, int batch = 1, long sA = 0, long sB = 0,
                  long sC = 0) {
    dim3 grid((N + 63) / 64, (unsigned)((M + 63) / 64), batch);
    k_sgemm<<<grid, 256, 0, st>>>((int)M, N, K, alpha, A, as0, as1, sA, B, bs0, bs1, sB, beta, C, ldc, sC, 0L);
}

// out[i] = sum over z of part[z][i], z in order
__global__ void k_sum_partials(int nz, long n, const float* __restrict__ part, float* __restrict__ out) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = 0.f;
    for (int z = 0; z < nz; ++z) v += part[(long)z * n + i];
    out[i] = v;
}

// A weight gradient C (M x N, contiguous) = op(A) op(B) over a long K (the point pairs of a batch):
// split-K over up to kMaxSplit chunks of at least 2048 pairs, so that the few output tiles still
// spread over the whole GPU; the partial products land in `part`, summed in chunk order.
constexpr int kMaxSplit = 256;
static void sgemm_wgrad(int M, int N, long K, const float* A, long as0, long as1, const float* B, long bs0, long bs1,
                        float* C, float* part, cudaStream_t st) {
    int nsplit = (int)((K + 2047) / 2048);
    if (nsplit > kMaxSplit) nsplit = kMaxSplit;
    if (nsplit < 1) nsplit = 1;
    const long kchunk = (K + nsplit - 1) / nsplit;
    nsplit = (int)((K + kchunk - 1) / kchunk);
    dim3 grid((N + 63) / 64, (unsigned)((M + 63) / 64), nsplit);
    k_sgemm<<<grid, 256, 0, st>>>(M, N, (int)K, 1.f, A, as0, as1, kchunk * as1, B, bs0, bs1, kchunk * bs0, 0.f, part,
                                  N, (long)M * N, kchunk);
    const long n = (long)M * N;
    k_sum_partials<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nsplit, n, part, C);
}

// ---------------------------------------------------------------------------
// features
// ---------------------------------------------------------------------------
// gbar[b][i] = mean of g[b][j] over the neighbours of i
__global__ void k_lpc_nbrmean(int B, int P, const float* __restrict__ g, const int* __restrict__ nbr,
                              const int* __restrict__ cnt, float* __restrict__ gbar) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * P) return;
    const int b = t / P, i = t % P, n = cnt[i];
    float s[4] = {0.f, 0.f, 0.f, 0.f};
    for (int q = 0; q < n; ++q) {
        const float* gj = g + ((size_t)b * P + nbr[i * 8 + q]) * 4;
        for (int c = 0; c < 4; ++c) s[c] += gj[c];
    }
    const float inv = n > 0 ? 1.f / n : 0.f;
    for (int c = 0; c < 4; ++c) gbar[(size_t)t * 4 + c] = s[c] * inv;
}

__device__ __forceinline__ void pair_features(const float* gi, const float* bi, const float* gj, const float* bj,
                                              float* x) {
    for (int c = 0; c < 4; ++c) {
        x[c] = gi[c];
        x[4 + c] = bi[c];
        x[8 + c] = gj[c];
        x[12 + c] = bj[c];
    }
    const float dx = gi[0] - gj[0], dy = gi[1] - gj[1];
    x[16] = dx;
    x[17] = dy;
    x[18] = sqrtf(dx * dx + dy * dy);
}

// X[(b P + i) P + j][19]
__global__ void k_lpc_pair_inputs(int B, int P, const float* __restrict__ g, const float* __restrict__ gbar,
                                  float* __restrict__ X) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)B * P * P) return;
    const int j = (int)(t % P);
    const long bi = t / P;
    const int i = (int)(bi % P), b = (int)(bi / P);
    const size_t pi = (size_t)b * P + i, pj = (size_t)b * P + j;
    pair_features(g + pi * 4, gbar + pi * 4, g + pj * 4, gbar + pj * 4, X + t * kF);
}

// y = relu(x + bias) in place on a rows x n matrix
__global__ void k_bias_relu(long total, int n, const float* __restrict__ bias, float* __restrict__ x) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const float v = x[t] + bias[t % n];
    x[t] = v > 0.f ? v : 0.f;
}

// K[b] = sym(Kraw) with Kraw[a P + i][c P + j] = KO[(b P + i) P + j][2a + c] + b3[2a + c]
__global__ void k_lpc_assemble_train(int B, int P, const float* __restrict__ KO, const float* __restrict__ b3,
                                     float* __restrict__ K) {
    const int m = 2 * P;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)B * m * m) return;
    const int col = (int)(t % m);
    const long br = t / m;
    const int row = (int)(br % m), b = (int)(br / m);
    auto raw = [&](int r, int c) {
        const int a = r / P, i = r % P, cc = c / P, j = c % P;
        return KO[(((size_t)b * P + i) * P + j) * kO + 2 * a + cc] + b3[2 * a + cc];
    };
    K[t] = 0.5f * (raw(row, col) + raw(col, row));
}

// E[b] -= I; loss per configuration sum(E^2) / m; E <- 2 E / (B m) (the loss gradient)
__global__ void k_lpc_residual_loss(int m, int B, float* __restrict__ E, float* __restrict__ lossc) {
    __shared__ float red[32];
    const int b = blockIdx.x;
    float* e = E + (size_t)b * m * m;
    float acc = 0.f;
    for (long t = threadIdx.x; t < (long)m * m; t += blockDim.x) {
        float v = e[t];
        if (t / m == t % m) v -= 1.f;
        acc += v * v;
        e[t] = 2.f * v / ((float)B * m);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        lossc[b] = s / m;
    }
}

// dKO[(b P + i) P + j][2a + c] = (dK[b][aP+i][cP+j] + dK[b][cP+j][aP+i]) / 2
__global__ void k_lpc_dko(int B, int P, const float* __restrict__ dK, float* __restrict__ dKO) {
    const int m = 2 * P;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)B * P * P * kO) return;
    const int q = (int)(t % kO);
    const long pair = t / kO;
    const int j = (int)(pair % P);
    const long bi = pair / P;
    const int i = (int)(bi % P), b = (int)(bi / P);
    const int a = q / 2, c = q % 2;
    const float* d = dK + (size_t)b * m * m;
    const int r = a * P + i, cc = c * P + j;
    dKO[t] = 0.5f * (d[(size_t)r * m + cc] + d[(size_t)cc * m + r]);
}

// dh *= (h > 0)
__global__ void k_relu_mask(long total, const float* __restrict__ h, float* __restrict__ dh) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < total && !(h[t] > 0.f)) dh[t] = 0.f;
}

// column sums of a rows x n matrix: one block per column, fixed summation order
__global__ void k_colsum(long rows, int n, const float* __restrict__ x, float* __restrict__ out) {
    __shared__ float red[32];
    const int c = blockIdx.x;
    float s = 0.f;
    for (long r = threadIdx.x; r < rows; r += blockDim.x) s += x[r * n + c];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        out[c] = t;
    }
}

__global__ void k_adam(long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, float lr, float b1, float b2, float c1, float c2, float eps) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    p[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// ---------------------------------------------------------------------------
// inference (one configuration, BF16 weights and activations)
// ---------------------------------------------------------------------------
// geometry features of the current body configuration: positions about each
// body's centroid over its extent, unit normals from the boundary neighbours
__global__ void k_lpc_geometry(int P, const double* __restrict__ pts, const int* __restrict__ body_of,
                               const int* __restrict__ body_start, const int* __restrict__ body_len,
                               const int* __restrict__ closed, float* __restrict__ g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const int bd = body_of[i], s0 = body_start[bd], n = body_len[bd];
    double cx = 0, cy = 0;
    for (int k = 0; k < n; ++k) {
        cx += pts[2 * (s0 + k)];
        cy += pts[2 * (s0 + k) + 1];
    }
    cx /= n;
    cy /= n;
    double ext = 1e-30;
    for (int k = 0; k < n; ++k) {
        const double dx = pts[2 * (s0 + k)] - cx, dy = pts[2 * (s0 + k) + 1] - cy;
        ext = fmax(ext, sqrt(dx * dx + dy * dy));
    }
    const int li = i - s0;
    int ip = li + 1, im = li - 1;
    if (closed[bd]) {
        ip = (ip + n) % n;
        im = (im + n) % n;
    } else {
        ip = min(ip, n - 1);
        im = max(im, 0);
    }
    const double tx = pts[2 * (s0 + ip)] - pts[2 * (s0 + im)], ty = pts[2 * (s0 + ip) + 1] - pts[2 * (s0 + im) + 1];
    const double tl = sqrt(tx * tx + ty * ty) + 1e-300;
    g[i * 4 + 0] = (float)((pts[2 * i] - cx) / ext);
    g[i * 4 + 1] = (float)((pts[2 * i + 1] - cy) / ext);
    g[i * 4 + 2] = (float)(ty / tl);
    g[i * 4 + 3] = (float)(-tx / tl);
}

constexpr int kPairsPerCta = 32;

// one CTA of 256 threads (thread = hidden unit) per 32 point pairs
__global__ void __launch_bounds__(256) k_lpc_pair_infer(int P, const float* __restrict__ g,
                                                        const float* __restrict__ gbar,
                                                        const __nv_bfloat16* __restrict__ W1,
                                                        const float* __restrict__ b1,
                                                        const __nv_bfloat16* __restrict__ W2t,
                                                        const float* __restrict__ b2,
                                                        const __nv_bfloat16* __restrict__ W3,
                                                        const float* __restrict__ b3, float* __restrict__ kraw) {
    __shared__ float X[kPairsPerCta][kF + 1];
    __shared__ float H[kPairsPerCta][kH + 1];
    const long npairs = (long)P * P;
    const long p0 = (long)blockIdx.x * kPairsPerCta;
    const int o = threadIdx.x;
    if (o < kPairsPerCta) {
        const long pr = p0 + o;
        if (pr < npairs) {
            const int i = (int)(pr / P), j = (int)(pr % P);
            pair_features(g + (size_t)i * 4, gbar + (size_t)i * 4, g + (size_t)j * 4, gbar + (size_t)j * 4, X[o]);
        } else {
            for (int c = 0; c < kF; ++c) X[o][c] = 0.f;
        }
    }
    __syncthreads();
    // layer 1
    {
        float w[kF];
        for (int c = 0; c < kF; ++c) w[c] = __bfloat162float(W1[o * kF + c]);
        const float bb = b1[o];
        for (int p = 0; p < kPairsPerCta; ++p) {
            float v = bb;
#pragma unroll
            for (int c = 0; c < kF; ++c) v += w[c] * X[p][c];
            H[p][o] = __bfloat162float(__float2bfloat16(v > 0.f ? v : 0.f));
        }
    }
    __syncthreads();
    // layer 2 (W2 stored transposed: W2t[k][o], coalesced over o)
    float acc[kPairsPerCta];
    {
        const float bb = b2[o];
#pragma unroll
        for (int p = 0; p < kPairsPerCta; ++p) acc[p] = bb;
        for (int k = 0; k < kH; ++k) {
            const float w = __bfloat162float(W2t[(size_t)k * kH + o]);
#pragma unroll
            for (int p = 0; p < kPairsPerCta; ++p) acc[p] += w * H[p][k];
        }
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < kPairsPerCta; ++p) H[p][o] = __bfloat162float(__float2bfloat16(acc[p] > 0.f ? acc[p] : 0.f));
    __syncthreads();
    // layer 3: 32 pairs x 4 outputs, one warp per 16 of them
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = warp; q < kPairsPerCta * kO; q += 8) {
        const int p = q / kO, c = q % kO;
        float v = 0.f;
        for (int k = lane; k < kH; k += 32) v += __bfloat162float(W3[c * kH + k]) * H[p][k];
        for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
        if (lane == 0 && p0 + p < npairs) kraw[(size_t)(p0 + p) * kO + c] = v + b3[c];
    }
}

// Kout[k][r][c] = (kraw(r, c) + kraw(c, r)) / (2 c0 beta_k) for every sub-step k
struct KOut {
    double* p[4];
    double s[4];
};
__global__ void k_lpc_assemble(int P, int nsub, const float* __restrict__ kraw, const float* __restrict__ c0p,
                               KOut out) {
    const int m = 2 * P;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)m * m) return;
    const int row = (int)(t / m), col = (int)(t % m);
    auto raw = [&](int r, int c) {
        const int a = r / P, i = r % P, cc = c / P, j = c % P;
        return (double)kraw[((size_t)i * P + j) * kO + 2 * a + cc];
    };
    const double v = 0.5 * (raw(row, col) + raw(col, row)) / (double)(*c0p);
    for (int k = 0; k < nsub; ++k) out.p[k][t] = v * out.s[k];
}

// BF16 copies: W1 as is, W2 transposed, W3 as is
__global__ void k_lpc_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ w) {
    const long n1 = (long)kH * kF, n2 = (long)kH * kH, n3 = (long)kO * kH;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n1) {
        w[t] = __float2bfloat16(p[oW1 + t]);
    } else if (t < n1 + n2) {
        const long u = t - n1, k = u / kH, o = u % kH;  // W2t[k][o] = W2[o][k]
        w[t] = __float2bfloat16(p[oW2 + o * kH + k]);
    } else if (t < n1 + n2 + n3) {
        w[t] = __float2bfloat16(p[oW3 + (t - n1 - n2)]);
    }
}

// ---------------------------------------------------------------------------
// host objects
// ---------------------------------------------------------------------------
int Lpc::init(int npts, const std::vector<int>& nbr_h, const std::vector<int>& cnt_h) {
    P = npts;
    const long w = (long)kH * kF + (long)kH * kH + (long)kO * kH;
    if (cudaMalloc(&params, sizeof(float) * kNParams) || cudaMalloc(&nbr, sizeof(int) * 8 * P) ||
        cudaMalloc(&cnt, sizeof(int) * P) || cudaMalloc(&wbf, sizeof(__nv_bfloat16) * w) ||
        cudaMalloc(&geom, sizeof(float) * 4 * P) || cudaMalloc(&gbar, sizeof(float) * 4 * P) ||
        cudaMalloc(&kraw, sizeof(float) * (size_t)P * P * kO) || cudaMalloc(&w2op, sizeof(__nv_bfloat16) * kH * kH) ||
        cudaMalloc(&err, sizeof(int)))
        return IBG_ERR_CUDA;
    cudaMemset(err, 0, sizeof(int));
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (lpc_infer_tc_setup()) return IBG_ERR_CUDA;
    cudaMemcpy(nbr, nbr_h.data(), sizeof(int) * 8 * P, cudaMemcpyHostToDevice);
    cudaMemcpy(cnt, cnt_h.data(), sizeof(int) * P, cudaMemcpyHostToDevice);
    // He initialisation with a fixed seed; the output layer starts small
    std::vector<float> h(kNParams, 0.f);
    std::mt19937 rng(1234);
    auto fill = [&](size_t off, int rows, int cols, float gain) {
        std::normal_distribution<float> nd(0.f, gain * std::sqrt(2.f / cols));
        for (int k = 0; k < rows * cols; ++k) h[off + k] = nd(rng);
    };
    fill(oW1, kH, kF, 1.f);
    fill(oW2, kH, kH, 1.f);
    fill(oW3, kO, kH, 0.1f);
    h[oC0] = 1.f;
    cudaMemcpy(params, h.data(), sizeof(float) * kNParams, cudaMemcpyHostToDevice);
    refresh_bf16(nullptr);
    return cudaDeviceSynchronize() == cudaSuccess ? IBG_OK : IBG_ERR_CUDA;
}

void Lpc::release() {
    void* p[] = {params, nbr, cnt, wbf, geom, gbar, kraw, w2op, err};
    for (void* x : p)
        if (x) cudaFree(x);
    params = nullptr;
    nbr = cnt = nullptr;
    wbf = w2op = nullptr;
    err = nullptr;
    geom = gbar = kraw = nullptr;
}

void Lpc::refresh_bf16(cudaStream_t st) {
    const long w = (long)kH * kF + (long)kH * kH + (long)kO * kH;
    k_lpc_to_bf16<<<(unsigned)((w + 255) / 256), 256, 0, st>>>(params, (__nv_bfloat16*)wbf);
    lpc_w2_operand(params, w2op, st);
}

void Lpc::geometry(const double* pts, const LpcBodies& bodies, cudaStream_t st) const {
    k_lpc_geometry<<<(P + 127) / 128, 128, 0, st>>>(P, pts, bodies.body_of, bodies.start, bodies.len, bodies.closed,
                                                    geom);
    k_lpc_nbrmean<<<(P + 127) / 128, 128, 0, st>>>(1, P, geom, nbr, cnt, gbar);
}

void Lpc::operators(int nsub, const double* beta, double* const* Kout, cudaStream_t st) const {
    const __nv_bfloat16* w = (const __nv_bfloat16*)wbf;
    const __nv_bfloat16* W1 = w;
    const __nv_bfloat16* W2t = W1 + (size_t)kH * kF;
    const __nv_bfloat16* W3 = W2t + (size_t)kH * kH;
    const long npairs = (long)P * P;
    if (tensor_cores)
        lpc_infer_tc(P, geom, gbar, params, w2op, kraw, err, num_sms, st);
    else
        k_lpc_pair_infer<<<(unsigned)((npairs + kPairsPerCta - 1) / kPairsPerCta), 256, 0, st>>>(
            P, geom, gbar, W1, params + oB1, W2t, params + oB2, W3, params + oB3, kraw);
    KOut o{};
    for (int k = 0; k < nsub && k < 4; ++k) {
        o.p[k] = Kout[k];
        o.s[k] = 1.0 / beta[k];
    }
    const long m2 = 4 * npairs;
    k_lpc_assemble<<<(unsigned)((m2 + 255) / 256), 256, 0, st>>>(P, nsub < 4 ? nsub : 4, kraw, params + oC0, o);
}

int Lpc::loss_grad(int B, const float* g, const float* Mb, float* loss, float* grad, TrainScratch& ws,
                   cudaStream_t st) const {
    const int m = 2 * P;
    const long rows = (long)B * P * P;
    if (ws.rows < rows || ws.cfgs < B) {
        ws.release();
        const size_t mm = (size_t)B * m * m;
        if (cudaMalloc(&ws.gbar, sizeof(float) * (size_t)B * P * 4) || cudaMalloc(&ws.X, sizeof(float) * rows * kF) ||
            cudaMalloc(&ws.H1, sizeof(float) * rows * kH) || cudaMalloc(&ws.H2, sizeof(float) * rows * kH) ||
            cudaMalloc(&ws.KO, sizeof(float) * rows * kO) || cudaMalloc(&ws.K, sizeof(float) * mm) ||
            cudaMalloc(&ws.E, sizeof(float) * mm) || cudaMalloc(&ws.dK, sizeof(float) * mm) ||
            cudaMalloc(&ws.dKO, sizeof(float) * rows * kO) || cudaMalloc(&ws.dH2, sizeof(float) * rows * kH) ||
            cudaMalloc(&ws.dH1, sizeof(float) * rows * kH) || cudaMalloc(&ws.lossc, sizeof(float) * B) ||
            cudaMalloc(&ws.part, sizeof(float) * (size_t)kMaxSplit * kH * kH)) {
            ws.release();
            return IBG_ERR_CUDA;
        }
        ws.rows = rows;
        ws.cfgs = B;
    }
    float c0 = 1.f;
    cudaMemcpyAsync(&c0, params + oC0, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return IBG_ERR_CUDA;
    const float* W1 = params + oW1;
    const float* W2 = params + oW2;
    const float* W3 = params + oW3;
    const long mm = (long)m * m;
    auto blocks = [](long n) { return (unsigned)((n + 255) / 256); };
    // forward
    k_lpc_nbrmean<<<(B * P + 127) / 128, 128, 0, st>>>(B, P, g, nbr, cnt, ws.gbar);
    k_lpc_pair_inputs<<<blocks(rows), 256, 0, st>>>(B, P, g, ws.gbar, ws.X);
    sgemm(rows, kH, kF, 1.f, ws.X, kF, 1, W1, 1, kF, 0.f, ws.H1, kH, st);
    k_bias_relu<<<blocks(rows * kH), 256, 0, st>>>(rows * kH, kH, params + oB1, ws.H1);
    sgemm(rows, kH, kH, 1.f, ws.H1, kH, 1, W2, 1, kH, 0.f, ws.H2, kH, st);
    k_bias_relu<<<blocks(rows * kH), 256, 0, st>>>(rows * kH, kH, params + oB2, ws.H2);
    sgemm(rows, kO, kH, 1.f, ws.H2, kH, 1, W3, 1, kH, 0.f, ws.KO, kO, st);
    k_lpc_assemble_train<<<blocks((long)B * mm), 256, 0, st>>>(B, P, ws.KO, params + oB3, ws.K);
    // E = K Mn - I with Mn = Mb / c0; loss; E <- dL/dE
    sgemm(m, m, m, 1.f / c0, ws.K, m, 1, Mb, m, 1, 0.f, ws.E, m, st, B, mm, mm, mm);
    k_lpc_residual_loss<<<B, 256, 0, st>>>(m, B, ws.E, ws.lossc);
    std::vector<float> lc(B);
    cudaMemcpyAsync(lc.data(), ws.lossc, sizeof(float) * B, cudaMemcpyDeviceToHost, st);
    if (grad) {
        // dK = dE Mn^T, then through the symmetrisation to the per-pair outputs
        sgemm(m, m, m, 1.f / c0, ws.E, m, 1, Mb, 1, m, 0.f, ws.dK, m, st, B, mm, mm, mm);
        k_lpc_dko<<<blocks(rows * kO), 256, 0, st>>>(B, P, ws.dK, ws.dKO);
        // layer 3: dW3 = dKO^T H2, db3, dH2 = dKO W3 (masked)
        sgemm_wgrad(kO, kH, rows, ws.dKO, 1, kO, ws.H2, kH, 1, grad + oW3, ws.part, st);
        k_colsum<<<kO, 256, 0, st>>>(rows, kO, ws.dKO, grad + oB3);
        sgemm(rows, kH, kO, 1.f, ws.dKO, kO, 1, W3, kH, 1, 0.f, ws.dH2, kH, st);
        k_relu_mask<<<blocks(rows * kH), 256, 0, st>>>(rows * kH, ws.H2, ws.dH2);
        // layer 2: dW2 = dH2^T H1, db2, dH1 = dH2 W2 (masked)
        sgemm_wgrad(kH, kH, rows, ws.dH2, 1, kH, ws.H1, kH, 1, grad + oW2, ws.part, st);
        k_colsum<<<kH, 256, 0, st>>>(rows, kH, ws.dH2, grad + oB2);
        sgemm(rows, kH, kH, 1.f, ws.dH2, kH, 1, W2, kH, 1, 0.f, ws.dH1, kH, st);
        k_relu_mask<<<blocks(rows * kH), 256, 0, st>>>(rows * kH, ws.H1, ws.dH1);
        // layer 1: dW1 = dH1^T X, db1
        sgemm_wgrad(kH, kF, rows, ws.dH1, 1, kH, ws.X, kF, 1, grad + oW1, ws.part, st);
        k_colsum<<<kH, 256, 0, st>>>(rows, kH, ws.dH1, grad + oB1);
        cudaMemsetAsync(grad + oC0, 0, sizeof(float), st);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return IBG_ERR_CUDA;
    if (loss) {
        double a = 0;
        for (float v : lc) a += v;
        *loss = (float)(a / B);
    }
    return IBG_OK;
}

void TrainScratch::release() {
    float* p[] = {gbar, X, H1, H2, KO, K, E, dK, dKO, dH2, dH1, lossc, part};
    for (float* x : p)
        if (x) cudaFree(x);
    gbar = X = H1 = H2 = KO = K = E = dK = dKO = dH2 = dH1 = lossc = part = nullptr;
    rows = 0;
    cfgs = 0;
}

void adam_step(long n, float* p, const float* g, float* m1, float* m2, float lr, int t, cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)t), c2 = 1.f - std::pow(b2, (float)t);
    k_adam<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, p, g, m1, m2, lr, b1, b2, c1, c2, 1e-8f);
}

}  // namespace ibg
