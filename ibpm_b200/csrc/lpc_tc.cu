// lpc_tc.cu -- inference of the learned preconditioner's network on the
// 5th-generation tensor cores (tcgen05, sm_100a).
//
// The network (lpc.cu) maps every ordered pair of boundary points to a 2 x 2
// block: 19 features -> 256 -> 256 -> 4 with ReLU.  Its 256 x 256 hidden layer
// over the P^2 pairs is the contraction: H2 = relu(H1 W2^T + b2) with H1 the
// (pairs x 256) first-layer activations.  One persistent CTA per SM keeps W2
// (BF16, 128 KiB) in shared memory and loops over tiles of 128 pairs:
//   1. the tile's first layer on the CUDA cores (8 warps; warp w computes the
//      128-unit half w / 4 of rows 32 (w % 4) ... + 31), rounded to BF16 and
//      written to shared memory as the MMA's A operand;
//   2. one thread issues sixteen tcgen05.mma kind::f16 (M = 128, N = 256,
//      K = 16 each) with the FP32 accumulator in tensor memory (256 columns),
//      then tcgen05.commit to an mbarrier;
//   3. every warp reads its lane quarter of the accumulator (tcgen05.ld),
//      adds b2, applies ReLU, rounds to BF16 (as the CUDA-core kernel does) and
//      contracts with the 4 x 256 last layer; the two halves of each row are
//      summed through shared memory and written as kraw[pair][4].
// Operands use the no-swizzle K-major layout of 8 x 16-byte core matrices:
// element (r, k) of a (rows x 256) BF16 operand at byte
// ((r / 8) * 32 + k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2, so adjacent core
// matrices along K are 128 bytes apart (leading byte offset) and adjacent
// 8-row groups 4096 bytes apart (stride byte offset).
// Every wait is bounded: an mbarrier wait that runs out sets *err, and the CTA
// releases its tensor memory and returns.
#include <cuda_bf16.h>

#include <cstdint>

#include "ibg_internal.cuh"
#include "ibg_lpc.cuh"

namespace ibg {

namespace {
constexpr int kF = 19, kH = 256, kO = 4;
constexpr int kRows = 128;                     // pairs per tile (MMA M)
constexpr int kTmemCols = 256;                 // FP32 accumulator columns (MMA N)
constexpr uint32_t kOffA = 0;                  // 128 x 256 BF16
constexpr uint32_t kOffB = kOffA + 65536;      // 256 x 256 BF16 (W2, rows = output units)
constexpr uint32_t kOffW1 = kOffB + 131072;    // 256 x 19 FP32 (BF16-rounded values)
constexpr uint32_t kOffB1 = kOffW1 + 4 * kH * kF;
constexpr uint32_t kOffB2 = kOffB1 + 4 * kH;
constexpr uint32_t kOffW3 = kOffB2 + 4 * kH;   // 4 x 256 FP32 (BF16-rounded values)
constexpr uint32_t kOffPart = kOffW3 + 4 * kO * kH;  // 128 rows x 4 partial outputs of the upper half
constexpr uint32_t kOffBar = kOffPart + 4 * kRows * kO;
constexpr uint32_t kOffTmem = kOffBar + 8;
constexpr uint32_t kSmemBytes = kOffTmem + 8;

// parameter offsets (floats), as lpc.cu lays them out
constexpr size_t oW1 = 0, oB1 = oW1 + (size_t)kH * kF, oW2 = oB1 + kH, oB2 = oW2 + (size_t)kH * kH,
                 oW3 = oB2 + kH, oB3 = oW3 + (size_t)kO * kH;

// byte offset of element (r, k) in a K-major no-swizzle operand with 256 columns
__host__ __device__ __forceinline__ uint32_t core_off(int r, int k) {
    return (uint32_t)((((r >> 3) * 32 + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// tcgen05 shared-memory matrix descriptor: start address, leading byte offset
// (K direction), stride byte offset (8-row groups), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)(128 >> 4) << 16;
    d |= (uint64_t)(4096 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, N, M
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTmemCols >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ float bf16_round(float v) { return __bfloat162float(__float2bfloat16(v)); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const uint32_t lo = (uint32_t)__bfloat16_as_ushort(__float2bfloat16(a));
    const uint32_t hi = (uint32_t)__bfloat16_as_ushort(__float2bfloat16(b));
    return lo | (hi << 16);
}

// waits for phase `parity` of the mbarrier; false when about 2^31 cycles pass first
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
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

__device__ __forceinline__ void pair_feat(const float* gi, const float* bi, const float* gj, const float* bj,
                                          float* x) {
#pragma unroll
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
}  // namespace

// W2 (FP32, [out][in]) as the MMA's B operand: BF16 in the core-matrix layout
__global__ void k_lpc_w2_operand(const float* __restrict__ params, __nv_bfloat16* __restrict__ w2op) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= kH * kH) return;
    const int n = t / kH, k = t % kH;
    w2op[core_off(n, k) >> 1] = __float2bfloat16(params[oW2 + (size_t)n * kH + k]);
}

__global__ void __launch_bounds__(256, 1) k_lpc_pair_infer_tc(int P, const float* __restrict__ g,
                                                              const float* __restrict__ gbar,
                                                              const float* __restrict__ params,
                                                              const __nv_bfloat16* __restrict__ w2op,
                                                              float* __restrict__ kraw, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quarter = warp & 3, half = warp >> 2;
    const int row = 32 * quarter + lane;
    float* W1s = (float*)(smem + kOffW1);
    float* b1s = (float*)(smem + kOffB1);
    float* b2s = (float*)(smem + kOffB2);
    float* W3s = (float*)(smem + kOffW3);
    float* part = (float*)(smem + kOffPart);
    const uint32_t sA = smem_u32(smem + kOffA), sB = smem_u32(smem + kOffB);
    const uint32_t bar = smem_u32(smem + kOffBar), tslot = smem_u32(smem + kOffTmem);

    // weights into shared memory (W2 as the B operand, the rest as BF16-rounded FP32)
    {
        const uint4* src = (const uint4*)w2op;
        uint4* dst = (uint4*)(smem + kOffB);
        for (int q = tid; q < kH * kH * 2 / 16; q += blockDim.x) dst[q] = src[q];
        for (int q = tid; q < kH * kF; q += blockDim.x) W1s[q] = bf16_round(params[oW1 + q]);
        for (int q = tid; q < kH; q += blockDim.x) {
            b1s[q] = params[oB1 + q];
            b2s[q] = params[oB2 + q];
        }
        for (int q = tid; q < kO * kH; q += blockDim.x) W3s[q] = bf16_round(params[oW3 + q]);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tslot),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *(volatile uint32_t*)(smem + kOffTmem);
    const float b3_0 = params[oB3], b3_1 = params[oB3 + 1], b3_2 = params[oB3 + 2], b3_3 = params[oB3 + 3];

    const long npairs = (long)P * P;
    const long ntiles = (npairs + kRows - 1) / kRows;
    uint32_t parity = 0;
    for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long pr = t * kRows + row;
        // 1. first layer of this thread's row, units [128 half, 128 half + 128)
        float x[kF];
        if (pr < npairs) {
            const int i = (int)(pr / P), j = (int)(pr % P);
            pair_feat(g + 4 * (size_t)i, gbar + 4 * (size_t)i, g + 4 * (size_t)j, gbar + 4 * (size_t)j, x);
        } else {
#pragma unroll
            for (int c = 0; c < kF; ++c) x[c] = 0.f;
        }
        for (int kc = 0; kc < 16; ++kc) {
            const int o0 = 128 * half + 8 * kc;
            uint32_t w4[4];
#pragma unroll
            for (int e = 0; e < 8; e += 2) {
                float v0 = b1s[o0 + e], v1 = b1s[o0 + e + 1];
#pragma unroll
                for (int c = 0; c < kF; ++c) {
                    v0 += W1s[(o0 + e) * kF + c] * x[c];
                    v1 += W1s[(o0 + e + 1) * kF + c] * x[c];
                }
                w4[e >> 1] = pack_bf16(v0 > 0.f ? v0 : 0.f, v1 > 0.f ? v1 : 0.f);
            }
            *(uint4*)(smem + kOffA + core_off(row, o0)) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
        }
        // make the generic-proxy writes of A visible to the tensor cores, then issue
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < kH / 16; ++s) {
                const uint64_t ad = smem_desc(sA + 256u * s), bd = smem_desc(sB + 256u * s);
                const uint32_t acc = s > 0 ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        const bool ok = mbar_wait_bounded(bar, parity);
        parity ^= 1u;
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(err, 1);
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // 3. epilogue: this warp's lane quarter, this half's 128 columns
        float o0 = 0.f, o1 = 0.f, o2 = 0.f, o3 = 0.f;
#pragma unroll 1
        for (int ch = 0; ch < 4; ++ch) {
            const int col = 128 * half + 32 * ch;
            const uint32_t taddr = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)col;
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
            for (int e = 0; e < 32; ++e) {
                const int k = col + e;
                float v = __uint_as_float(r[e]) + b2s[k];
                v = bf16_round(v > 0.f ? v : 0.f);
                o0 += W3s[k] * v;
                o1 += W3s[kH + k] * v;
                o2 += W3s[2 * kH + k] * v;
                o3 += W3s[3 * kH + k] * v;
            }
        }
        if (half == 1) {
            part[4 * row] = o0;
            part[4 * row + 1] = o1;
            part[4 * row + 2] = o2;
            part[4 * row + 3] = o3;
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (half == 0 && pr < npairs) {
            float4 out;
            out.x = o0 + part[4 * row] + b3_0;
            out.y = o1 + part[4 * row + 1] + b3_1;
            out.z = o2 + part[4 * row + 2] + b3_2;
            out.w = o3 + part[4 * row + 3] + b3_3;
            *(float4*)(kraw + 4 * pr) = out;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
}

int lpc_infer_tc_setup() {
    static bool done = false;
    if (done) return IBG_OK;
    if (cudaFuncSetAttribute(k_lpc_pair_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes) !=
        cudaSuccess)
        return IBG_ERR_CUDA;
    done = true;
    return IBG_OK;
}

void lpc_w2_operand(const float* params, void* w2op, cudaStream_t st) {
    k_lpc_w2_operand<<<(kH * kH + 255) / 256, 256, 0, st>>>(params, (__nv_bfloat16*)w2op);
}

void lpc_infer_tc(int P, const float* g, const float* gbar, const float* params, const void* w2op, float* kraw,
                  int* err, int num_sms, cudaStream_t st) {
    const long ntiles = ((long)P * P + kRows - 1) / kRows;
    const int grid = (int)(ntiles < num_sms ? ntiles : num_sms);
    k_lpc_pair_infer_tc<<<grid, 256, kSmemBytes, st>>>(P, g, gbar, params, (const __nv_bfloat16*)w2op, kraw, err);
}

}  // namespace ibg
