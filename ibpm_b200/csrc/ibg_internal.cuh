// ibg_internal.cuh -- shared definitions for the B200 IBPM time step.
//
// Device layouts are the reference's own (so state moves between host and
// device without reshuffling):
//   Scalar  [batch][lev][i-1][j-1]           (nx-1)(ny-1) values per level
//   Flux    [batch][lev][index]              x-fluxes i*ny+j, then y-fluxes
//                                            at (nx+1)*ny + i*(ny+1)+j
//   Bndry   [fx_0..fx_{n-1}, fy_0..fy_{n-1}]
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <utility>
#include <cstdlib>

namespace ibg {

// Raise a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device.  The limit is a property of the function, shared by every
// context in the process, so it only ever grows (a context with a smaller grid
// must not lower the limit another context's launches rely on).
int raise_smem_limit(const void* func, int bytes);

// ---------------------------------------------------------------------------
// grid description passed by value to kernels
// ---------------------------------------------------------------------------
struct GridDev {
    int nx, ny, L;          // cells per level, number of levels
    int nxe, nye;           // coarse cells left of / below the finer domain
    int NI, NJ;             // interior nodes per row / column: nx-1, ny-1
    int N1;                 // nodes per level (nx-1)(ny-1)
    int nXf;                // x-fluxes per level (nx+1) ny
    int F1;                 // fluxes per level
    double dx;              // finest spacing
    double x0, y0;          // lower-left corner of level 0
};

__host__ __device__ inline double lev_dx(const GridDev& g, int lev) { return g.dx * (double)(1 << lev); }

// ---------------------------------------------------------------------------
// Programmatic dependent launch.  Kernels of the time step are launched with
// launch_k, which lets the next kernel on the stream be scheduled while the
// one ahead of it is still running; every such kernel starts with
// pdl_enter(): it waits until the kernels it depends on have finished and
// their writes are visible (griddepcontrol.wait, before any global memory
// access), then allows the kernel after it to be scheduled
// (griddepcontrol.launch_dependents).  For a kernel launched without the
// attribute both are no-ops.  IBG_PDL=0 in the environment turns the
// attribute off.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

bool pdl_enabled();

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                            Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// value of a Scalar level at node (i, j), 1 <= i <= nx-1, 1 <= j <= ny-1
template <typename T>
__device__ __forceinline__ T node(const T* lev_base, const GridDev& g, int i, int j) {
    return lev_base[(size_t)(i - 1) * g.NJ + (j - 1)];
}

// Boundary ring values of level `lev` taken from the next coarser level `c`
// (the coarse level's interior array).  Coincident nodes copy, in-between
// nodes average (reference Scalar::getBC, src/Scalar.cc:91-127).
template <typename T>
__device__ __forceinline__ T bc_bottom(const T* c, const GridDev& g, int i) {
    int ii = i / 2 + g.nxe, jj = g.nye;
    T a = node(c, g, ii, jj);
    if (i & 1) return (T)0.5 * (a + node(c, g, ii + 1, jj));
    return a;
}
template <typename T>
__device__ __forceinline__ T bc_top(const T* c, const GridDev& g, int i) {
    int ii = i / 2 + g.nxe, jj = g.ny / 2 + g.nye;
    T a = node(c, g, ii, jj);
    if (i & 1) return (T)0.5 * (a + node(c, g, ii + 1, jj));
    return a;
}
template <typename T>
__device__ __forceinline__ T bc_left(const T* c, const GridDev& g, int j) {
    int ii = g.nxe, jj = j / 2 + g.nye;
    T a = node(c, g, ii, jj);
    if (j & 1) return (T)0.5 * (a + node(c, g, ii, jj + 1));
    return a;
}
template <typename T>
__device__ __forceinline__ T bc_right(const T* c, const GridDev& g, int j) {
    int ii = g.nx / 2 + g.nxe, jj = j / 2 + g.nye;
    T a = node(c, g, ii, jj);
    if (j & 1) return (T)0.5 * (a + node(c, g, ii, jj + 1));
    return a;
}

// Node value with the boundary ring filled from `coarse` (nullptr: zeros),
// for 0 <= i <= nx, 0 <= j <= ny.
template <typename T>
__device__ __forceinline__ T node_bc(const T* f, const T* coarse, const GridDev& g, int i, int j) {
    if (i >= 1 && i <= g.nx - 1 && j >= 1 && j <= g.ny - 1) return node(f, g, i, j);
    if (coarse == nullptr) return (T)0;
    if (j == 0) return bc_bottom(coarse, g, i);
    if (j == g.ny) return bc_top(coarse, g, i);
    if (i == 0) return bc_left(coarse, g, j);
    return bc_right(coarse, g, j);
}

// ---------------------------------------------------------------------------
// FFT descriptor for one complex length m = 2 (n + 1)
// ---------------------------------------------------------------------------
constexpr int kMaxFactors = 24;
constexpr int kMaxRadix = 16;
struct FftDesc {
    int m;
    int nfac;
    int fac[kMaxFactors];
    const void* tw;  // m complex twiddles w_m^k (double2 or float2)
};

// ---------------------------------------------------------------------------
// error reporting
// ---------------------------------------------------------------------------
enum Status {
    IBG_OK = 0,
    IBG_ERR_ARG = -1,
    IBG_ERR_CUDA = -2,
    IBG_ERR_UNSUPPORTED = -3,
    IBG_ERR_STATE = -4,
    IBG_ERR_IO = -5,
    IBG_ERR_NOT_CONVERGED = -6,
    IBG_ERR_NUMERIC = -7,
};

}  // namespace ibg
