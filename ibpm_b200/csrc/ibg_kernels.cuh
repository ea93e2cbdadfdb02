// ibg_kernels.cuh -- kernel argument blocks and host-side plan objects.
#pragma once
#include "ibg_internal.cuh"

namespace ibg {

template <typename T>
struct RowPassArgs {
    GridDev g;
    FftDesc fft;
    int pairs_per_block;
    const T* in;
    size_t in_bstride;       // batch stride of `in` and `coarse`
    T* out;
    size_t out_bstride;      // batch stride of `out`, `out2`, `base`
    T* out2;                 // optional: out2 = base - out
    const T* base;
    int lift;                // apply in_scale and boundary lifting on load
    T in_scale;
    const T* coarse;         // next coarser solution level (nullptr: zero boundary)
    T bc_coef;
    T norm;                  // output scale
};

template <typename T>
struct ColPassArgs {
    GridDev g;
    FftDesc fft;
    int pairs_per_block;
    T* buf;
    size_t bstride;
    const T* cosx;
    const T* cosy;
    T bydx2;
    int helmholtz;
    T alpha;
};

struct FftTables {
    FftDesc row64{}, col64{}, row32{}, col32{};
    void* tw_row64 = nullptr;
    void* tw_row32 = nullptr;
    void* tw_col64 = nullptr;
    void* tw_col32 = nullptr;
    int init(int m_rows, int m_cols);
    void release();
};

struct CosTables {
    double* x64 = nullptr;
    double* y64 = nullptr;
    float* x32 = nullptr;
    float* y32 = nullptr;
    int init(int nx, int ny);
    void release();
};

bool fft_supported(int m);
// factor m into the radices the shared-memory FFT uses (no device allocation)
void fft_describe(int m, FftDesc& d);

// One multi-domain solve call.  All arrays are device pointers.
template <typename T>
struct SolveCall {
    const T* f;       // right-hand side, all levels
    T* u;             // solution, all levels
    T* rc;            // scratch: coarsified right-hand side (levels 1..L-1)
    T* tbuf;          // scratch: one level per batch item (N1 * batch)
    size_t bstride;   // batch stride of f, u, rc, out2, base
    int batch;
    T in_scale;       // multiplies the right-hand side (+1 or -1)
    T* out2;          // optional: out2 = base - u
    const T* base;
};

template <typename T>
struct EllipticPlan {
    const GridDev* grid = nullptr;
    const FftTables* tables = nullptr;
    int helmholtz = 0;
    double alpha = 0.0;
    int rows_pairs = 1, cols_pairs = 1, threads = 128;
    const double* cos64x = nullptr;
    const double* cos64y = nullptr;
    const float* cos32x = nullptr;
    const float* cos32y = nullptr;
    int init(const GridDev* g, const FftTables* t, bool helm, double a, const CosTables& ct);
    int solve(const SolveCall<T>& c, cudaStream_t st) const;
    // one pass of the finest level alone (0: rows of pass A, 1: columns of pass B), for timing
    void run_pass(int which, const T* in, T* tbuf, cudaStream_t st) const;
};

}  // namespace ibg
