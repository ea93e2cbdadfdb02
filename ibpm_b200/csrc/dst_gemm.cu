// dst_gemm.cu -- the DST-I passes of the FP32 multi-domain solves as sine-matrix
// GEMMs on the 5th-generation tensor cores (tcgen05, kind::tf32, 3xTF32).
//
// The reference transforms with FFTW's RODFT00 (src/EllipticSolver2d.cc:57-85):
// along a line of n values, Y_k = 2 sum_j X_j sin(pi (j+1)(k+1) / (n+1)), i.e.
// Y = S X with the symmetric n x n sine matrix S.  For the 2-D transform of a
// level (NI x NJ nodes, j contiguous):
//   rows    T[i][k] = sum_j X[i][j] S_y[j][k]      (A = X,   B = S_y)
//   columns U[i][k] = sum_i' S_x[i][i'] T[i'][k]   (A = S_x, B = T^T)
// so each pass is one GEMM per level.  This is the alternative to the
// shared-memory FFT passes (elliptic.cu); the autotuner picks one per grid.
//
// Precision: FP32 data, 3xTF32 products: every operand x is split into
// hi = tf32(x) and lo = tf32(x - hi), and A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi
// is accumulated in FP32 in tensor memory, which keeps FP32 accuracy (the
// dropped A_lo B_lo term is ~2^-22 relative).
//
// One CTA computes a 128 x NT tile of one level (NT <= 256 output columns,
// a multiple of 32), looping over K in chunks of 32 with two shared-memory
// stages.  All 256 threads hold the next chunk's operands in registers (its
// global loads are issued before the current chunk's MMAs), store them as
// float4s in the no-swizzle K-major core-matrix layout (each warp's stores fill
// 512 contiguous bytes, so no bank conflicts), and split the data operand into
// hi and lo in place, one item at a time; one thread issues 12 tcgen05.mma per
// chunk (4 K-steps of 8, 3 products each) and commits them to the stage's
// mbarrier.  Each mode is its own instantiation, so a kernel carries only its
// mode's code (the first version, one kernel for all modes with every staging
// loop unrolled, spent most of its time waiting for instruction fetches).  The
// epilogue reads the accumulator (tcgen05.ld), stages it through shared memory
// and stores it coalesced.  Every mbarrier wait is bounded: a wait that runs out
// sets *err and the CTA frees its tensor memory and returns.
//
// Modes (matching the FFT passes' steps of EllipticPlan::solve):
//   0  rows forward:  in (the overlap interior from alt) * in_scale -> out
//   1  rows inverse:  out = norm * (tbuf S_y), out2 = base - out
//   2  columns forward: src -> dst
//   3  columns inverse: the boundary lifting and eigen-inverse applied to the
//      coefficients as they are loaded, src -> dst
#include <cstdint>
#include <cstring>
#include <vector>

#include "ibg_internal.cuh"
#include "ibg_kernels.cuh"

namespace ibg {

namespace {
constexpr int kM = 128;        // rows per tile (MMA M)
constexpr int kKc = 32;        // K per chunk
constexpr int kThreads = 256;
constexpr uint32_t kAbytes = kM * kKc * 4;           // 16 KiB: one of A_hi / A_lo
constexpr uint32_t kBbytesMax = 256 * kKc * 4;       // 32 KiB: one of B_hi / B_lo at NT = 256
constexpr uint32_t kStage = 2 * kAbytes + 2 * kBbytesMax;  // 96 KiB
constexpr uint32_t kOffBar = 2 * kStage;             // two mbarriers
constexpr uint32_t kOffTmem = kOffBar + 16;
constexpr uint32_t kSmem = kOffTmem + 16;

// byte offset of element (r, k) of a K-major no-swizzle TF32 operand chunk with 32 K values:
// 8 x 16-byte core matrices, 8 along K (128 bytes apart), 8-row groups 1024 bytes apart
__device__ __forceinline__ uint32_t core32(int r, int k) {
    return (uint32_t)((((r >> 3) << 3) + (k >> 2)) << 7) + (uint32_t)((r & 7) << 4) + (uint32_t)((k & 3) << 2);
}

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)(128 >> 4) << 16;   // leading byte offset: next core matrix along K
    d |= (uint64_t)(1024 >> 4) << 32;  // stride byte offset: next 8-row group
    d |= (uint64_t)1 << 46;            // descriptor version
    return d;
}

// kind::tf32 instruction descriptor: FP32 accumulator, TF32 A and B, K-major both, N, M = 128
__device__ __forceinline__ uint32_t idesc_tf32(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
}

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__device__ __forceinline__ bool wait_bounded(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > (1LL << 31)) return false;
    }
}

__device__ __forceinline__ bool in_overlap(const GridDev& g, int i, int j) {
    return i > g.nxe && i < g.nx / 2 + g.nxe && j > g.nye && j < g.ny / 2 + g.nye;
}
}  // namespace

// Operand staging.  A K-major operand tile of R rows x 32 K values is cut into items of 8 rows x 16 K;
// in an item, lane l takes row 8 rg + (l & 7) and the four K values 16 kh + 4 (l >> 3) .. + 3, so a
// warp's float4 stores fill four consecutive core matrices (512 contiguous bytes, no bank conflict)
// and its global reads of a row-major operand cover 8 rows x 64 bytes (or, for the transposed T,
// 4 rows of T x 32 bytes).
constexpr int kAItems = (kM / 8) * 2;  // 32 items: 4 per warp

__device__ __forceinline__ void item_pos(int item, int lane, int& r, int& k) {
    r = 8 * (item >> 1) + (lane & 7);
    k = 16 * (item & 1) + 4 * (lane >> 3);
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, 1) k_dst_gemm(GemmPassArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    pdl_enter();
    constexpr bool ROWS = MODE <= 1;
    constexpr int kBmaxPer = 256 / 32;  // B items per warp at NT = 256
    const GridDev& g = a.g;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int NT = a.n_tile;  // a multiple of 32
    const int Mdim = g.NI, Ndim = g.NJ, Kdim = ROWS ? g.NJ : g.NI;
    const int b = blockIdx.z / a.nlev, lev = blockIdx.z % a.nlev;
    const int m0 = blockIdx.x * kM, n0 = blockIdx.y * NT;
    const int nchunks = (Kdim + kKc - 1) / kKc;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t bar0 = sbase + kOffBar, bar1 = bar0 + 8, tslot = sbase + kOffTmem;
    const uint32_t Bbytes = (uint32_t)NT * kKc * 4;
    const int bper = NT / 32;  // B items per warp

    const float* X = nullptr;  // rows passes: the level's data (A)
    const float* Xalt = nullptr;
    const float* T = nullptr;  // columns passes: the level's coefficients (B = T^T)
    const float* edges = nullptr;
    if (ROWS) {
        X = a.in[lev] + (size_t)b * a.in_bstride;
        Xalt = a.alt[lev] ? a.alt[lev] + (size_t)b * a.in_bstride : nullptr;
    } else {
        T = a.src + (size_t)b * a.bstride + (size_t)lev * a.lstride;
        if (MODE == 3 && a.edges && lev < a.nlev - 1) edges = a.edges + (size_t)b * a.estride + (size_t)lev * a.elstride;
    }
    const float bydx2 = a.bydx2[lev], bcc = a.bc_coef[lev];

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tslot),
                     "r"(a.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *(volatile uint32_t*)(smem + kOffTmem);
    const uint32_t idesc = idesc_tf32(NT);

    // registers of the next chunk: the data operand (raw) and the sine operand (hi, lo)
    float dv[kBmaxPer > 4 ? kBmaxPer * 4 : 16];       // rows: A data (4 items); columns: B data (bper items)
    float sh[kBmaxPer * 4], sl[kBmaxPer * 4];           // rows: B = S_y (bper items); columns: A = S_x (4 items)
    auto load = [&](int c) {
        const int k0 = c * kKc;
        if (ROWS) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                int r, k;
                item_pos(warp * 4 + q, lane, r, k);
                const int gr = m0 + r;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int gk = k0 + k + j;
                    float v = 0.f;
                    if (gr < Mdim && gk < Kdim) {
                        const float* src = (Xalt && in_overlap(g, gr + 1, gk + 1)) ? Xalt : X;
                        v = src[(size_t)gr * Ndim + gk];
                    }
                    dv[4 * q + j] = v;
                }
            }
#pragma unroll
            for (int q = 0; q < kBmaxPer; ++q) {
                if (q >= bper) break;
                int r, k;
                item_pos(warp * bper + q, lane, r, k);
                const int gn = n0 + r;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int gk = k0 + k + j;
                    const bool in = gn < Ndim && gk < Kdim;
                    sh[4 * q + j] = in ? a.s_hi[(size_t)gn * Kdim + gk] : 0.f;
                    sl[4 * q + j] = in ? a.s_lo[(size_t)gn * Kdim + gk] : 0.f;
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                int r, k;
                item_pos(warp * 4 + q, lane, r, k);
                const int gr = m0 + r;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int gk = k0 + k + j;
                    const bool in = gr < Mdim && gk < Kdim;
                    sh[4 * q + j] = in ? a.s_hi[(size_t)gr * Kdim + gk] : 0.f;
                    sl[4 * q + j] = in ? a.s_lo[(size_t)gr * Kdim + gk] : 0.f;
                }
            }
#pragma unroll
            for (int q = 0; q < kBmaxPer; ++q) {
                if (q >= bper) break;
                int r, k;
                item_pos(warp * bper + q, lane, r, k);
                const int gn = n0 + r;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int gk = k0 + k + j;
                    dv[4 * q + j] = (gn < Ndim && gk < Kdim) ? T[(size_t)gk * Ndim + gn] : 0.f;
                }
            }
        }
    };
    // registers -> stage st: the sine operand as loaded, the data operand raw into its hi area, then
    // (one item at a time, not unrolled) scaled / lifted and split into hi and lo in place
    auto store = [&](int c, int st) {
        unsigned char* S0 = smem + (size_t)st * kStage;
        unsigned char* Ahi = S0;
        unsigned char* Alo = S0 + kAbytes;
        unsigned char* Bhi = S0 + 2 * kAbytes;
        unsigned char* Blo = Bhi + Bbytes;
        unsigned char* Dhi = ROWS ? Ahi : Bhi;  // the data operand
        unsigned char* Dlo = ROWS ? Alo : Blo;
        unsigned char* Shi = ROWS ? Bhi : Ahi;  // the sine operand
        unsigned char* Slo = ROWS ? Blo : Alo;
        const int nd = ROWS ? 4 : bper, ns = ROWS ? bper : 4;
        const int dbase = ROWS ? warp * 4 : warp * bper, sbase_ = ROWS ? warp * bper : warp * 4;
#pragma unroll
        for (int q = 0; q < kBmaxPer; ++q) {
            if (q >= ns) break;
            int r, k;
            item_pos(sbase_ + q, lane, r, k);
            *(float4*)(Shi + core32(r, k)) = make_float4(sh[4 * q], sh[4 * q + 1], sh[4 * q + 2], sh[4 * q + 3]);
            *(float4*)(Slo + core32(r, k)) = make_float4(sl[4 * q], sl[4 * q + 1], sl[4 * q + 2], sl[4 * q + 3]);
        }
#pragma unroll
        for (int q = 0; q < kBmaxPer; ++q) {
            if (q >= nd) break;
            int r, k;
            item_pos(dbase + q, lane, r, k);
            *(float4*)(Dhi + core32(r, k)) = make_float4(dv[4 * q], dv[4 * q + 1], dv[4 * q + 2], dv[4 * q + 3]);
        }
        const int k0 = c * kKc;
#pragma unroll 1
        for (int q = 0; q < nd; ++q) {
            int r, k;
            item_pos(dbase + q, lane, r, k);
            float4 v = *(float4*)(Dhi + core32(r, k));
            float e[4] = {v.x, v.y, v.z, v.w}, hi[4], lo[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float x = e[j];
                if (ROWS) {
                    x = a.in_scale * x;
                } else if (MODE == 3) {
                    const int gn = n0 + r, gk = k0 + k + j;
                    if (gn < Ndim && gk < Kdim)
                        x = lifted_coef(x, gk, gn, edges, Mdim, Ndim, bcc, a.s, a.cosx, a.cosy, bydx2, a.helmholtz,
                                        a.alpha);
                }
                hi[j] = tf32_rna(x);
                lo[j] = tf32_rna(x - hi[j]);
            }
            *(float4*)(Dhi + core32(r, k)) = make_float4(hi[0], hi[1], hi[2], hi[3]);
            *(float4*)(Dlo + core32(r, k)) = make_float4(lo[0], lo[1], lo[2], lo[3]);
        }
    };

    bool ok = true;
    uint32_t ph[2] = {0u, 0u};
    load(0);
    for (int c = 0; c < nchunks; ++c) {
        const int st = c & 1;
        if (c >= 2) {
            // the MMAs of chunk c - 2 read this stage: wait for them before overwriting it
            ok = wait_bounded(st ? bar1 : bar0, ph[st]);
            ph[st] ^= 1u;
            if (__syncthreads_or(!ok)) break;
        }
        store(c, st);
        if (c + 1 < nchunks) load(c + 1);  // in flight while this chunk is issued
        // make this stage's generic-proxy writes visible to the tensor cores, then issue
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            const uint32_t S0 = sbase + (uint32_t)st * kStage;
            const uint32_t Ahi = S0, Alo = S0 + kAbytes, Bhi = S0 + 2 * kAbytes, Blo = Bhi + Bbytes;
#pragma unroll
            for (int ks = 0; ks < kKc / 8; ++ks) {
                const uint32_t o = 256u * ks;
                const uint64_t dAh = sdesc(Ahi + o), dAl = sdesc(Alo + o), dBh = sdesc(Bhi + o), dBl = sdesc(Blo + o);
                const uint64_t ad[3] = {dAh, dAh, dAl}, bd[3] = {dBh, dBl, dBh};
#pragma unroll
                for (int p = 0; p < 3; ++p) {
                    const uint32_t acc = (c > 0 || ks > 0 || p > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n .reg .pred q;\n setp.ne.b32 q, %4, 0;\n"
                        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, q;\n}\n" ::"r"(tmem),
                        "l"(ad[p]), "l"(bd[p]), "r"(idesc), "r"(acc)
                        : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             st ? bar1 : bar0)
                         : "memory");
        }
    }
    if (ok) {
        // the last chunk's MMAs complete the accumulator (and every earlier one, in issue order);
        // the other stage's last commit is waited for too, so that no arrival is left pending
        const int lst = (nchunks - 1) & 1;
        ok = wait_bounded(lst ? bar1 : bar0, ph[lst]);
        if (nchunks >= 2) {
            const int other = lst ^ 1;
            ok = ok && wait_bounded(other ? bar1 : bar0, ph[other]);
        }
    }
    if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicExch(a.err, 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // epilogue: accumulator rows through shared memory (the stages are free now), then coalesced stores
        float* Dt = (float*)smem;  // [128][NT + 1]
        const int ld = NT + 1;
        const int quarter = warp & 3, half = warp >> 2;
        const int row = 32 * quarter + lane;
        for (int c0 = half * 32; c0 < NT; c0 += 64) {
            const uint32_t taddr = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)c0;
            uint32_t r[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                "[%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(taddr)
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int e = 0; e < 32; ++e) Dt[row * ld + c0 + e] = __uint_as_float(r[e]);
        }
        __syncthreads();
        const int ncols = min(NT, Ndim - n0);
        const int nrows = min(kM, Mdim - m0);
        for (int e = tid; e < nrows * NT; e += kThreads) {
            const int rr = e / NT, cc = e - rr * NT;
            if (cc >= ncols) continue;
            const size_t gi = (size_t)(m0 + rr) * Ndim + (n0 + cc);
            const float v = Dt[rr * ld + cc];
            if (MODE == 0) {
                a.out[lev][(size_t)b * a.out_bstride + gi] = v;
            } else if (MODE == 1) {
                const float u = v * a.norm;
                a.out[lev][(size_t)b * a.out_bstride + gi] = u;
                if (a.out2[lev]) a.out2[lev][(size_t)b * a.out_bstride + gi] = a.base[lev][(size_t)b * a.out_bstride + gi] - u;
            } else {
                a.dst[(size_t)b * a.bstride + (size_t)lev * a.lstride + gi] = v;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols)
                     : "memory");
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {
// TF32 round to nearest, ties away from zero (cvt.rna), in host arithmetic
float tf32_host(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u = (u + 0x1000u) & 0xFFFFE000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}
}  // namespace

int SineMats::init(int nx, int ny) {
    const double pi = 3.14159265358979323846264338327950288;
    auto make = [&](int n, float** hi, float** lo) -> int {
        std::vector<float> h((size_t)n * n), l((size_t)n * n);
        for (int a = 0; a < n; ++a)
            for (int c = 0; c < n; ++c) {
                // (a + 1)(c + 1) reduced mod 2 (n + 1) keeps the sine's argument small and exact
                const long q = ((long)(a + 1) * (c + 1)) % (2L * (n + 1));
                const double s = 2.0 * sin(pi * (double)q / (double)(n + 1));
                const float f = (float)s;
                const float fh = tf32_host(f);
                h[(size_t)a * n + c] = fh;
                l[(size_t)a * n + c] = tf32_host((float)(s - (double)fh));
            }
        if (cudaMalloc(hi, sizeof(float) * h.size()) != cudaSuccess ||
            cudaMalloc(lo, sizeof(float) * l.size()) != cudaSuccess)
            return IBG_ERR_CUDA;
        cudaMemcpy(*hi, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(*lo, l.data(), sizeof(float) * l.size(), cudaMemcpyHostToDevice);
        return IBG_OK;
    };
    if (make(nx - 1, &sx_hi, &sx_lo) || make(ny - 1, &sy_hi, &sy_lo)) return IBG_ERR_CUDA;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return IBG_ERR_CUDA;
    cudaMemset(err, 0, sizeof(int));
    return IBG_OK;
}

void SineMats::release() {
    float* p[] = {sx_hi, sx_lo, sy_hi, sy_lo};
    for (float* x : p)
        if (x) cudaFree(x);
    if (err) cudaFree(err);
    sx_hi = sx_lo = sy_hi = sy_lo = nullptr;
    err = nullptr;
}

int gemm_pass_setup() {
    static bool done = false;
    if (done) return IBG_OK;
    const void* fns[4] = {(const void*)k_dst_gemm<0>, (const void*)k_dst_gemm<1>, (const void*)k_dst_gemm<2>,
                          (const void*)k_dst_gemm<3>};
    for (const void* f : fns)
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem) != cudaSuccess)
            return IBG_ERR_CUDA;
    done = true;
    return IBG_OK;
}

void launch_gemm_pass(GemmPassArgs& a, int batch, cudaStream_t st) {
    const GridDev& g = a.g;
    const int N = g.NJ;
    // at least four column tiles per level, so that small levels still spread over several SMs;
    // a multiple of 32 (whole staging items per warp), at most 256 (one MMA)
    int nt = (((N + 3) / 4) + 31) / 32 * 32;
    nt = nt < 32 ? 32 : nt > 256 ? 256 : nt;
    a.n_tile = nt;
    a.tmem_cols = nt <= 32 ? 32 : nt <= 64 ? 64 : nt <= 128 ? 128 : 256;
    const dim3 grid((unsigned)((g.NI + kM - 1) / kM), (unsigned)((N + nt - 1) / nt), (unsigned)(a.nlev * batch));
    switch (a.mode) {
        case 0: launch_k(k_dst_gemm<0>, grid, kThreads, (size_t)kSmem, st, a); break;
        case 1: launch_k(k_dst_gemm<1>, grid, kThreads, (size_t)kSmem, st, a); break;
        case 2: launch_k(k_dst_gemm<2>, grid, kThreads, (size_t)kSmem, st, a); break;
        default: launch_k(k_dst_gemm<3>, grid, kThreads, (size_t)kSmem, st, a); break;
    }
}

}  // namespace ibg
