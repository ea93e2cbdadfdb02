// lpc.cu -- learned preconditioner for the moving-body force solve.
//
// A network over the boundary points maps a CG residual r to z ~ M^-1 r,
// used as the preconditioner of the flexible CG (the reference has no
// counterpart; it runs plain CG, src/ConjugateGradientSolver.cc:35-65).
//
//   input per point i:  a_i = (x, y, nx, ny, rx/s, ry/s), s = rms(r),
//                       x, y about the body centroid over its extent,
//                       (nx, ny) the unit normal from the neighbours
//   layer 1:            h1_i = relu(W1 [a_i | mean_{j in N(i)} a_j] + b1)      12 -> 256
//   layer 2:            h2_i = relu(W2 [h1_i | mean_{j in N(i)} h1_j] + b2)   512 -> 256
//   layer 3:            o_i  = W3 h2_i + b3                                    256 -> 2
//   output:             z_i  = (s / beta) o_i
// N(i) are up to 8 neighbours along the body (i +- 1..4, wrapping on closed
// bodies).  The factor s makes P(c r) = c P(r) for c > 0; 1/beta carries the
// sub-step scale of M = beta C A^-1 B.
//
// Training (FP32): loss = mean over samples of |o - t|^2 / |t|^2 with targets
// t = beta z / s, gradients by hand-written backward kernels, Adam.
// Inference (BF16 weights and hidden activations, FP32 accumulation).
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
constexpr int kIn = 6, kIn2 = 12, kH = 256, kH2 = 512, kOut = 2;
constexpr size_t oW1 = 0, oB1 = oW1 + (size_t)kH * kIn2, oW2 = oB1 + kH, oB2 = oW2 + (size_t)kH * kH2,
                 oW3 = oB2 + kH, oB3 = oW3 + (size_t)kOut * kH, kNParams = oB3 + kOut;

size_t lpc_num_params() { return kNParams; }

// ---------------------------------------------------------------------------
// generic FP32 GEMM: C[M x N] = alpha op(A) op(B) + beta C, element (i, k) of
// op(A) at A[i * as0 + k * as1], (k, j) of op(B) at B[k * bs0 + j * bs1].
// 64 x 64 tiles, 256 threads, 4 x 4 outputs per thread.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, float alpha, const float* __restrict__ A,
                                               long as0, long as1, const float* __restrict__ B, long bs0, long bs1,
                                               float beta, float* __restrict__ C, long ldc) {
    __shared__ float As[16][64 + 1];
    __shared__ float Bs[16][64 + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int i0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int t = threadIdx.x; t < 16 * 64; t += 256) {
            const int kk = t / 64, ii = t % 64;
            const int gi = i0 + ii, gk = k0 + kk;
            As[kk][ii] = (gi < M && gk < K) ? A[gi * as0 + gk * as1] : 0.f;
            const int gj = j0 + ii;
            Bs[kk][ii] = (gk < K && gj < N) ? B[gk * bs0 + gj * bs1] : 0.f;
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
        const int gi = i0 + ty * 4 + r;
        if (gi >= M) continue;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int gj = j0 + tx * 4 + c;
            if (gj >= N) continue;
            float v = alpha * acc[r][c];
            if (beta != 0.f) v += beta * C[gi * ldc + gj];
            C[gi * ldc + gj] = v;
        }
    }
}

static void sgemm(int M, int N, int K, float alpha, const float* A, long as0, long as1, const float* B, long bs0,
                  long bs1, float beta, float* C, long ldc, cudaStream_t st) {
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    k_sgemm<<<grid, 256, 0, st>>>(M, N, K, alpha, A, as0, as1, B, bs0, bs1, beta, C, ldc);
}

// ---------------------------------------------------------------------------
// training kernels (rows = samples x points, row = b * P + i)
// ---------------------------------------------------------------------------
// per-sample residual scale s = rms(r) (one block per sample)
__global__ void k_lpc_scale(int P, const float* __restrict__ r, float* __restrict__ s) {
    __shared__ float red[32];
    const int b = blockIdx.x;
    float acc = 0.f;
    for (int k = threadIdx.x; k < 2 * P; k += blockDim.x) {
        const float v = r[(size_t)b * 2 * P + k];
        acc += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        s[b] = sqrtf(t / (2 * P)) + 1e-30f;
    }
}

// A = [a_i | mean_nbr a_j] (rows x 12); geometry per sample g[b][i][4], residual r[b][2P] as [x.. | y..]
__global__ void k_lpc_inputs(int P, int rows, const float* __restrict__ g, const float* __restrict__ r,
                             const float* __restrict__ s, const int* __restrict__ nbr, const int* __restrict__ cnt,
                             float* __restrict__ A) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= rows) return;
    const int b = row / P, i = row % P;
    auto feat = [&](int j, float* f) {
        const float* gg = g + ((size_t)b * P + j) * 4;
        f[0] = gg[0]; f[1] = gg[1]; f[2] = gg[2]; f[3] = gg[3];
        f[4] = r[(size_t)b * 2 * P + j] / s[b];
        f[5] = r[(size_t)b * 2 * P + P + j] / s[b];
    };
    float own[kIn], mean[kIn] = {0, 0, 0, 0, 0, 0};
    feat(i, own);
    const int n = cnt[i];
    for (int q = 0; q < n; ++q) {
        float f[kIn];
        feat(nbr[i * 8 + q], f);
        for (int c = 0; c < kIn; ++c) mean[c] += f[c];
    }
    const float inv = n > 0 ? 1.f / n : 0.f;
    float* a = A + (size_t)row * kIn2;
    for (int c = 0; c < kIn; ++c) {
        a[c] = own[c];
        a[kIn + c] = mean[c] * inv;
    }
}

// y = relu(x + bias) in place on a rows x n matrix
__global__ void k_bias_relu(long total, int n, const float* __restrict__ bias, float* __restrict__ x) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const float v = x[t] + bias[t % n];
    x[t] = v > 0.f ? v : 0.f;
}

// C = [h1_i | mean_nbr h1_j] (rows x 512)
__global__ void k_lpc_concat(int P, int rows, const float* __restrict__ h1, const int* __restrict__ nbr,
                             const int* __restrict__ cnt, float* __restrict__ C) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)rows * kH) return;
    const int row = (int)(t / kH), o = (int)(t % kH);
    const int b = row / P, i = row % P;
    const int n = cnt[i];
    float m = 0.f;
    for (int q = 0; q < n; ++q) m += h1[((size_t)b * P + nbr[i * 8 + q]) * kH + o];
    C[(size_t)row * kH2 + o] = h1[(size_t)row * kH + o];
    C[(size_t)row * kH2 + kH + o] = n > 0 ? m / n : 0.f;
}

// output layer, per-sample loss and dL/do (one block per sample)
__global__ void k_lpc_out_loss(int P, int B, const float* __restrict__ h2, const float* __restrict__ W3,
                               const float* __restrict__ b3, const float* __restrict__ t, float* __restrict__ out,
                               float* __restrict__ dout, float* __restrict__ loss_per_sample) {
    __shared__ float red[32];
    const int b = blockIdx.x;
    // |t_b|^2
    float tt = 0.f;
    for (int k = threadIdx.x; k < 2 * P; k += blockDim.x) {
        const float v = t[(size_t)b * 2 * P + k];
        tt += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) tt += __shfl_xor_sync(0xffffffffu, tt, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = tt;
    __syncthreads();
    float tsum = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tsum += red[w];
    __syncthreads();
    const float denom = tsum + 1e-12f;
    float el = 0.f;
    for (int q = threadIdx.x; q < 2 * P; q += blockDim.x) {
        const int c = q / P, i = q % P;  // component, point
        const float* h = h2 + ((size_t)b * P + i) * kH;
        float o = b3[c];
        for (int k = 0; k < kH; ++k) o += W3[c * kH + k] * h[k];
        const float e = o - t[(size_t)b * 2 * P + c * P + i];
        out[((size_t)b * P + i) * 2 + c] = o;
        dout[((size_t)b * P + i) * 2 + c] = 2.f * e / (denom * B);
        el += e * e;
    }
    for (int o = 16; o > 0; o >>= 1) el += __shfl_xor_sync(0xffffffffu, el, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = el;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        loss_per_sample[b] = s / denom;
    }
}

// dh = (dY W) masked by (h > 0): dh[row][o] = (sum_c dY[row][c] W[c][o]) (h[row][o] > 0), for the 2-output layer
__global__ void k_lpc_back3(long rows, const float* __restrict__ dout, const float* __restrict__ W3,
                            const float* __restrict__ h2, float* __restrict__ dh2) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= rows * kH) return;
    const long row = t / kH;
    const int o = (int)(t % kH);
    const float g = dout[row * 2] * W3[o] + dout[row * 2 + 1] * W3[kH + o];
    dh2[t] = h2[t] > 0.f ? g : 0.f;
}

// dh1_i = (dC_i[:256] + sum_{j in N(i)} dC_j[256:] / |N(j)|) masked by h1 > 0
__global__ void k_lpc_back_concat(int P, int rows, const float* __restrict__ dC, const int* __restrict__ nbr,
                                  const int* __restrict__ cnt, const float* __restrict__ h1, float* __restrict__ dh1) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)rows * kH) return;
    const int row = (int)(t / kH), o = (int)(t % kH);
    const int b = row / P, i = row % P;
    float g = dC[(size_t)row * kH2 + o];
    const int n = cnt[i];
    for (int q = 0; q < n; ++q) {
        const int j = nbr[i * 8 + q];
        g += dC[((size_t)b * P + j) * kH2 + kH + o] / cnt[j];
    }
    dh1[t] = h1[t] > 0.f ? g : 0.f;
}

// column sums of a rows x n matrix into out[n] (+= scale * sum), deterministic order
__global__ void k_colsum(int rows, int n, const float* __restrict__ x, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    float s = 0.f;
    for (int r = 0; r < rows; ++r) s += x[(size_t)r * n + c];
    out[c] = s;
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
// inference kernels (one sample = the current boundary, BF16 weights)
// ---------------------------------------------------------------------------
// geometry features of the current body configuration: positions about each
// body's centroid over its extent, unit normals from the boundary neighbours
__global__ void k_lpc_geometry(int P, int nbodies, const double* __restrict__ pts, const int* __restrict__ body_of,
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
    (void)nbodies;
}

// z = (s / beta) net(r): one CTA of 256 threads per 8 points for layers 1-2,
// with the scale computed in the first phase of every CTA
__global__ void __launch_bounds__(256) k_lpc_infer_l1(int P, const double* __restrict__ r,
                                                      const float* __restrict__ g, const int* __restrict__ nbr,
                                                      const int* __restrict__ cnt,
                                                      const __nv_bfloat16* __restrict__ W1,
                                                      const float* __restrict__ b1, __nv_bfloat16* __restrict__ h1,
                                                      float* __restrict__ s_out) {
    __shared__ float red[8];
    __shared__ float s_sh;
    __shared__ float A[8][kIn2];
    // residual scale
    float acc = 0.f;
    for (int k = threadIdx.x; k < 2 * P; k += blockDim.x) acc += (float)(r[k] * r[k]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < 8; ++w) t += red[w];
        s_sh = sqrtf(t / (2 * P)) + 1e-30f;
        if (blockIdx.x == 0) *s_out = s_sh;
    }
    __syncthreads();
    const float s = s_sh;
    const int i0 = blockIdx.x * 8;
    if (threadIdx.x < 8 && i0 + threadIdx.x < P) {
        const int i = i0 + threadIdx.x;
        auto feat = [&](int j, float* f) {
            f[0] = g[j * 4]; f[1] = g[j * 4 + 1]; f[2] = g[j * 4 + 2]; f[3] = g[j * 4 + 3];
            f[4] = (float)r[j] / s;
            f[5] = (float)r[P + j] / s;
        };
        float own[kIn], mean[kIn] = {0, 0, 0, 0, 0, 0};
        feat(i, own);
        const int n = cnt[i];
        for (int q = 0; q < n; ++q) {
            float f[kIn];
            feat(nbr[i * 8 + q], f);
            for (int c = 0; c < kIn; ++c) mean[c] += f[c];
        }
        for (int c = 0; c < kIn; ++c) {
            A[threadIdx.x][c] = own[c];
            A[threadIdx.x][kIn + c] = n > 0 ? mean[c] / n : 0.f;
        }
    }
    __syncthreads();
    const int o = threadIdx.x;  // 256 outputs
    for (int pi = 0; pi < 8 && i0 + pi < P; ++pi) {
        float v = b1[o];
        for (int c = 0; c < kIn2; ++c) v += __bfloat162float(W1[o * kIn2 + c]) * A[pi][c];
        h1[(size_t)(i0 + pi) * kH + o] = __float2bfloat16(v > 0.f ? v : 0.f);
    }
}

__global__ void __launch_bounds__(256) k_lpc_infer_l2(int P, const int* __restrict__ nbr, const int* __restrict__ cnt,
                                                      const __nv_bfloat16* __restrict__ h1,
                                                      const __nv_bfloat16* __restrict__ W2,
                                                      const float* __restrict__ b2, __nv_bfloat16* __restrict__ h2) {
    __shared__ float Cs[4][kH2];
    const int i0 = blockIdx.x * 4;
    for (int t = threadIdx.x; t < 4 * kH; t += blockDim.x) {
        const int pi = t / kH, o = t % kH, i = i0 + pi;
        float own = 0.f, m = 0.f;
        if (i < P) {
            own = __bfloat162float(h1[(size_t)i * kH + o]);
            const int n = cnt[i];
            for (int q = 0; q < n; ++q) m += __bfloat162float(h1[(size_t)nbr[i * 8 + q] * kH + o]);
            if (n > 0) m /= n;
        }
        Cs[pi][o] = own;
        Cs[pi][kH + o] = m;
    }
    __syncthreads();
    const int o = threadIdx.x;
    float acc[4];
    for (int pi = 0; pi < 4; ++pi) acc[pi] = b2[o];
    const __nv_bfloat16* w = W2 + (size_t)o * kH2;
    for (int c = 0; c < kH2; ++c) {
        const float wv = __bfloat162float(w[c]);
#pragma unroll
        for (int pi = 0; pi < 4; ++pi) acc[pi] += wv * Cs[pi][c];
    }
    for (int pi = 0; pi < 4 && i0 + pi < P; ++pi)
        h2[(size_t)(i0 + pi) * kH + o] = __float2bfloat16(acc[pi] > 0.f ? acc[pi] : 0.f);
}

__global__ void k_lpc_infer_l3(int P, const __nv_bfloat16* __restrict__ h2, const __nv_bfloat16* __restrict__ W3,
                               const float* __restrict__ b3, const float* __restrict__ s, double inv_beta,
                               double* __restrict__ z) {
    const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= 2 * P) return;
    const int c = q / P, i = q % P;
    float acc = 0.f;
    for (int k = lane; k < kH; k += 32) acc += __bfloat162float(W3[c * kH + k]) * __bfloat162float(h2[(size_t)i * kH + k]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) z[c * P + i] = (double)(acc + b3[c]) * (double)(*s) * inv_beta;
}

__global__ void k_to_bf16(long n, const float* __restrict__ x, __nv_bfloat16* __restrict__ y) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

// ---------------------------------------------------------------------------
// host objects
// ---------------------------------------------------------------------------
int Lpc::init(int npts, const std::vector<int>& nbr_h, const std::vector<int>& cnt_h) {
    P = npts;
    if (cudaMalloc(&params, sizeof(float) * kNParams) || cudaMalloc(&nbr, sizeof(int) * 8 * P) ||
        cudaMalloc(&cnt, sizeof(int) * P) || cudaMalloc(&wbf, sizeof(__nv_bfloat16) * kNParams) ||
        cudaMalloc(&h1, sizeof(__nv_bfloat16) * (size_t)P * kH) ||
        cudaMalloc(&h2, sizeof(__nv_bfloat16) * (size_t)P * kH) || cudaMalloc(&geom, sizeof(float) * 4 * P) ||
        cudaMalloc(&scale, sizeof(float)))
        return IBG_ERR_CUDA;
    cudaMemcpy(nbr, nbr_h.data(), sizeof(int) * 8 * P, cudaMemcpyHostToDevice);
    cudaMemcpy(cnt, cnt_h.data(), sizeof(int) * P, cudaMemcpyHostToDevice);
    // He initialisation, fixed seed
    std::vector<float> h(kNParams, 0.f);
    std::mt19937 rng(1234);
    auto fill = [&](size_t off, int rows, int cols) {
        std::normal_distribution<float> nd(0.f, std::sqrt(2.f / cols));
        for (int k = 0; k < rows * cols; ++k) h[off + k] = nd(rng);
    };
    fill(oW1, kH, kIn2);
    fill(oW2, kH, kH2);
    fill(oW3, kOut, kH);
    for (int k = 0; k < kOut * kH; ++k) h[oW3 + k] *= 0.1f;
    cudaMemcpy(params, h.data(), sizeof(float) * kNParams, cudaMemcpyHostToDevice);
    refresh_bf16(nullptr);
    return IBG_OK;
}

void Lpc::release() {
    void* p[] = {params, nbr, cnt, wbf, h1, h2, geom, scale};
    for (void* x : p)
        if (x) cudaFree(x);
    params = nullptr;
    nbr = cnt = nullptr;
    wbf = nullptr;
    h1 = h2 = nullptr;
    geom = scale = nullptr;
}

void Lpc::refresh_bf16(cudaStream_t st) {
    k_to_bf16<<<(unsigned)((kNParams + 255) / 256), 256, 0, st>>>((long)kNParams, params, (__nv_bfloat16*)wbf);
}

void Lpc::apply(const double* pts, const LpcBodies& bodies, const double* r, double* z, double beta,
                cudaStream_t st) const {
    const __nv_bfloat16* w = (const __nv_bfloat16*)wbf;
    k_lpc_geometry<<<(P + 127) / 128, 128, 0, st>>>(P, bodies.n, pts, bodies.body_of, bodies.start, bodies.len,
                                                    bodies.closed, geom);
    k_lpc_infer_l1<<<(P + 7) / 8, 256, 0, st>>>(P, r, geom, nbr, cnt, w + oW1, params + oB1, (__nv_bfloat16*)h1,
                                                 scale);
    k_lpc_infer_l2<<<(P + 3) / 4, 256, 0, st>>>(P, nbr, cnt, (const __nv_bfloat16*)h1, w + oW2, params + oB2,
                                                 (__nv_bfloat16*)h2);
    k_lpc_infer_l3<<<(2 * P + 7) / 8, 256, 0, st>>>(P, (const __nv_bfloat16*)h2, w + oW3, params + oB3, scale,
                                                     1.0 / beta, z);
}

// one forward (and backward when grad != nullptr) pass over B samples held on the device
int Lpc::loss_grad(int B, const float* g, const float* r, const float* t, float* loss_per_sample, float* grad,
                   TrainScratch& ws, cudaStream_t st) const {
    const int rows = B * P;
    if (ws.rows < rows) {
        ws.release();
        if (cudaMalloc(&ws.A, sizeof(float) * (size_t)rows * kIn2) || cudaMalloc(&ws.s, sizeof(float) * B) ||
            cudaMalloc(&ws.h1, sizeof(float) * (size_t)rows * kH) ||
            cudaMalloc(&ws.C, sizeof(float) * (size_t)rows * kH2) ||
            cudaMalloc(&ws.h2, sizeof(float) * (size_t)rows * kH) ||
            cudaMalloc(&ws.out, sizeof(float) * (size_t)rows * 2) ||
            cudaMalloc(&ws.dout, sizeof(float) * (size_t)rows * 2) ||
            cudaMalloc(&ws.dh2, sizeof(float) * (size_t)rows * kH) ||
            cudaMalloc(&ws.dC, sizeof(float) * (size_t)rows * kH2) ||
            cudaMalloc(&ws.dh1, sizeof(float) * (size_t)rows * kH))
            return IBG_ERR_CUDA;
        ws.rows = rows;
    }
    const float* W1 = params + oW1;
    const float* W2 = params + oW2;
    const float* W3 = params + oW3;
    // forward
    k_lpc_scale<<<B, 256, 0, st>>>(P, r, ws.s);
    k_lpc_inputs<<<(rows + 127) / 128, 128, 0, st>>>(P, rows, g, r, ws.s, nbr, cnt, ws.A);
    sgemm(rows, kH, kIn2, 1.f, ws.A, kIn2, 1, W1, 1, kIn2, 0.f, ws.h1, kH, st);
    k_bias_relu<<<(unsigned)(((long)rows * kH + 255) / 256), 256, 0, st>>>((long)rows * kH, kH, params + oB1, ws.h1);
    k_lpc_concat<<<(unsigned)(((long)rows * kH + 255) / 256), 256, 0, st>>>(P, rows, ws.h1, nbr, cnt, ws.C);
    sgemm(rows, kH, kH2, 1.f, ws.C, kH2, 1, W2, 1, kH2, 0.f, ws.h2, kH, st);
    k_bias_relu<<<(unsigned)(((long)rows * kH + 255) / 256), 256, 0, st>>>((long)rows * kH, kH, params + oB2, ws.h2);
    k_lpc_out_loss<<<B, 256, 0, st>>>(P, B, ws.h2, W3, params + oB3, t, ws.out, ws.dout, loss_per_sample);
    if (!grad) return IBG_OK;
    // backward
    // dW3 = dout^T h2 (2 x 256), db3 = column sums of dout
    sgemm(kOut, kH, rows, 1.f, ws.dout, 1, 2, ws.h2, kH, 1, 0.f, grad + oW3, kH, st);
    k_colsum<<<1, 32, 0, st>>>(rows, kOut, ws.dout, grad + oB3);
    k_lpc_back3<<<(unsigned)(((long)rows * kH + 255) / 256), 256, 0, st>>>((long)rows, ws.dout, W3, ws.h2, ws.dh2);
    // dW2 = dh2^T C (256 x 512), db2, dC = dh2 W2 (rows x 512)
    sgemm(kH, kH2, rows, 1.f, ws.dh2, 1, kH, ws.C, kH2, 1, 0.f, grad + oW2, kH2, st);
    k_colsum<<<(kH + 127) / 128, 128, 0, st>>>(rows, kH, ws.dh2, grad + oB2);
    sgemm(rows, kH2, kH, 1.f, ws.dh2, kH, 1, W2, kH2, 1, 0.f, ws.dC, kH2, st);
    k_lpc_back_concat<<<(unsigned)(((long)rows * kH + 255) / 256), 256, 0, st>>>(P, rows, ws.dC, nbr, cnt, ws.h1,
                                                                                ws.dh1);
    // dW1 = dh1^T A (256 x 12), db1
    sgemm(kH, kIn2, rows, 1.f, ws.dh1, 1, kH, ws.A, kIn2, 1, 0.f, grad + oW1, kIn2, st);
    k_colsum<<<(kH + 127) / 128, 128, 0, st>>>(rows, kH, ws.dh1, grad + oB1);
    return cudaPeekAtLastError() == cudaSuccess ? IBG_OK : IBG_ERR_CUDA;
}

void TrainScratch::release() {
    float* p[] = {A, s, h1, C, h2, out, dout, dh2, dC, dh1};
    for (float* x : p)
        if (x) cudaFree(x);
    A = s = h1 = C = h2 = out = dout = dh2 = dC = dh1 = nullptr;
    rows = 0;
}

void adam_step(long n, float* p, const float* g, float* m1, float* m2, float lr, int t, cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)t), c2 = 1.f - std::pow(b2, (float)t);
    k_adam<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, p, g, m1, m2, lr, b1, b2, c1, c2, 1e-8f);
}

}  // namespace ibg
