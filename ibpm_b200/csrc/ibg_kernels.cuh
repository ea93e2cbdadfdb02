// ibg_kernels.cuh -- kernel argument blocks and host-side plan objects of the
// multi-domain elliptic solves.
#pragma once
#include <algorithm>
#include <memory>
#include <vector>

#include "ibg_internal.cuh"

namespace ibg {

constexpr int kMaxLevels = 16;
constexpr int kSweepRows = 4;    // coefficient rows per row-sum block of the sweep
constexpr int kSweepCols = 4;    // coefficient columns per column-sum block of the sweep

template <typename T>
struct RowPassArgs {
    GridDev g;
    FftDesc fft;
    int pairs_per_block;
    int tw_smem;                   // 1: twiddles copied to shared memory first
    int nlev;                      // levels in this launch: blockIdx.y = batch * nlev + level
    const T* in[kMaxLevels];       // per-level input (batch item 0)
    const T* alt[kMaxLevels];      // per-level input inside the overlap interior (nullptr: none)
    size_t in_bstride;
    T* out[kMaxLevels];
    size_t out_bstride;            // batch stride of out, out2, base
    T* out2[kMaxLevels];           // optional: out2 = base - out
    const T* base[kMaxLevels];
    T in_scale;                    // multiplies the input (+1 or -1)
    T norm;                        // multiplies the output
    const T* sinh;                 // sin(pi j / N), the half-length DST's pre-processing
};

// sine vectors (mode k + 1) of the spectral boundary lifting and the boundary lines
template <typename T>
struct SineTab {
    const T* sx1;   // 2 sin(pi K / nx)
    const T* sxn;   // 2 sin(pi (nx-1) K / nx)
    const T* si0;   // 2 sin(pi i0 K / nx), i0 = nxe
    const T* si1;   // 2 sin(pi i1 K / nx), i1 = nx/2 + nxe
    const T* sy1;
    const T* syn;
    const T* sj0;   // j0 = nye
    const T* sj1;   // j1 = ny/2 + nye
};

template <typename T>
struct ColPassArgs {
    GridDev g;
    FftDesc fft;
    int pairs_per_block;
    int tw_smem;                   // 1: twiddles copied to shared memory first
    int mode;                      // 0, 2: one DST along i; 1: DST, eigen-inverse, DST (one level);
                                   // 3: boundary lifting + eigen-inverse on load, one DST
    int nlev;
    T* buf;
    size_t lstride, bstride;       // level and batch strides
    const T* cosx;
    const T* cosy;
    SineTab<T> s;
    T bydx2[kMaxLevels];
    T bc_coef[kMaxLevels];
    int helmholtz;
    T alpha;
    const T* edges;                // boundary DSTs of every level (mode 3)
    size_t estride, elstride;      // batch and level strides of edges
    const T* sinh;                 // sin(pi j / N), the half-length DST's pre-processing
};


template <typename T>
struct GridTables {
    const T* cosx = nullptr;   // cos(pi i / nx), i < nx (FP32 tables: cos(pi i / nx) - 1)
    const T* cosy = nullptr;
    SineTab<T> s{};
    // edge maps of the coarse-to-fine sweep (row-major NI x NI and NJ x NJ; nullptr: FFT path)
    const T* ax = nullptr;
    const T* ay = nullptr;
};

template <typename T>
struct SweepArgs {
    GridDev g;
    FftDesc frow;                  // length 2 ny
    FftDesc fcol;                  // length 2 nx
    FftDesc frowh;                 // length ny: the half-length DSTs of k_sweep_lines (FP64, half = 1)
    FftDesc fcolh;                 // length nx
    int half;                      // the lines' DSTs by the half-length FFTs (else the odd extension)
    const T* sinr;                 // their pre-processing sines
    const T* sinc;
    const T* buf;                  // this level's forward coefficients (batch item 0)
    size_t bstride;
    const T* cosx;
    const T* cosy;
    SineTab<T> s;
    T bydx2;
    int helmholtz;
    T alpha;
    T bc_coef;                     // 1/dx^2 (Poisson) or alpha/dx^2 (Helmholtz) of this level
    const T* edges_in;             // this level's boundary DSTs (nullptr on the coarsest level)
    T* edges_out;                  // boundary DSTs of the next finer level
    size_t estride;                // batch stride of the edges arrays
    T* vrow;                       // work: row sums V0, V1 [NI] then column sums W0, W1 [NJ]
    size_t wstride;
    T norm;
    const T* ax;                   // edge maps (k_sweep_edges)
    const T* ay;
    int* counters;                 // 2 counters: the lines step runs inside k_sweep_sums (nullptr: its own launch)
};

// eigenvalue of the inverse operator at 0-based mode (k, l):
// lambda = 2 (cos(pi (k+1)/nx) + cos(pi (l+1)/ny) - 2) / dx^2 (src/EllipticSolver2d.cc:42-54),
// 1/lambda (Poisson, :115-122) or 1/(1 + alpha lambda) (Helmholtz, :156-163)
// The FP64 tables hold the cosines and lambda is formed as the reference forms it; the FP32 tables hold
// cos - 1 (tabulated in double as -2 sin^2(theta / 2)), because in float cos + cos - 2 cancels for the
// low modes: at n = 512 the lowest eigenvalue would lose three digits and the forces ~1e-4.
template <typename T>
__device__ __forceinline__ T eig_inverse(const T* cx, const T* cy, int k, int l, T bydx2, int helm, T alpha) {
    const T lam = sizeof(T) == 8 ? (T)2 * (cx[k + 1] + cy[l + 1] - (T)2) * bydx2 : (T)2 * (cx[k + 1] + cy[l + 1]) * bydx2;
    return helm ? (T)1 / ((T)1 + alpha * lam) : (T)1 / lam;
}

// Coefficient (k, l) of a level after the boundary lifting and the eigen-inverse:
// U = E (R - c Slift), Slift = sy1 B(k) + syn T(k) + sx1 L(l) + sxn R(l), where
// B, T, L, R are the 1-D DSTs of the level's bottom, top, left, right boundary values.
template <typename T>
__device__ __forceinline__ T lifted_coef(T R, int k, int l, const T* edges, int NI, int NJ, T c,
                                         const SineTab<T>& s, const T* cx, const T* cy, T bydx2, int helm,
                                         T alpha) {
    if (edges) {
        const T sl = s.sy1[l] * edges[k] + s.syn[l] * edges[NI + k] + s.sx1[k] * edges[2 * NI + l] +
                     s.sxn[k] * edges[2 * NI + NJ + l];
        R = R - c * sl;
    }
    return R * eig_inverse(cx, cy, k, l, bydx2, helm, alpha);
}

// ---------------------------------------------------------------------------
// sine-matrix GEMM form of the FP32 DST passes (dst_gemm.cu)
// ---------------------------------------------------------------------------
// the sine matrices S_x (NI x NI) and S_y (NJ x NJ), S[a][c] = 2 sin(pi (a+1)(c+1) / (n+1)),
// split into TF32 hi and lo parts (row-major FP32 arrays)
struct SineMats {
    float *sx_hi = nullptr, *sx_lo = nullptr, *sy_hi = nullptr, *sy_lo = nullptr;
    int* err = nullptr;  // set by a GEMM pass whose bounded wait ran out
    int init(int nx, int ny);
    void release();
};

struct GemmPassArgs {
    GridDev g;
    int mode;        // 0 rows forward, 1 rows inverse, 2 columns forward, 3 columns inverse (lifting + eigen-inverse)
    int nlev;
    int n_tile, tmem_cols;
    // rows passes: A = the level's data, B = S_y
    const float* in[kMaxLevels];
    const float* alt[kMaxLevels];
    size_t in_bstride;
    float* out[kMaxLevels];
    float* out2[kMaxLevels];
    const float* base[kMaxLevels];
    size_t out_bstride;
    float in_scale, norm;
    // columns passes: A = S_x, B = the level's coefficients transposed
    const float* src;
    float* dst;
    size_t lstride, bstride;
    const float* edges;
    size_t estride, elstride;
    const float* cosx;
    const float* cosy;
    SineTab<float> s;
    float bydx2[kMaxLevels];
    float bc_coef[kMaxLevels];
    int helmholtz;
    float alpha;
    const float* s_hi;   // the pass's sine matrix
    const float* s_lo;
    int* err;
};
int gemm_pass_setup();
void launch_gemm_pass(GemmPassArgs& a, int batch, cudaStream_t st);

struct FftTables {
    // length 2 (n + 1): the odd-extension FFTs of the sweep's boundary lines and the edge maps
    FftDesc row64{}, col64{}, row32{}, col32{};
    void* tw_row64 = nullptr;
    void* tw_row32 = nullptr;
    void* tw_col64 = nullptr;
    void* tw_col32 = nullptr;
    // length n + 1: the half-length DSTs of the FP64 row and column passes, with their
    // pre-processing sines sin(pi j / (n + 1)), j = 0 .. (n + 1) / 2
    FftDesc rowh64{}, colh64{};
    void *tw_rowh64 = nullptr, *tw_colh64 = nullptr;
    void *sin_row64 = nullptr, *sin_col64 = nullptr;
    int init(int m_rows, int m_cols);
    void release();
};
// the half-length DSTs' pre-processing sines of a precision (rows: pass 0, columns: pass 1; FP64 only)
template <typename T>
inline const T* pass_sines(const FftTables& t, int pass) {
    return sizeof(T) == 8 ? (const T*)(pass == 0 ? t.sin_row64 : t.sin_col64) : nullptr;
}

// doubles in one grid's table block: cos x, cos y, 4 x-sine vectors, 4 y-sine vectors
inline size_t table_doubles(int nx, int ny) { return (size_t)nx + ny + 4 * (size_t)(nx - 1) + 4 * (size_t)(ny - 1); }
void fill_grid_tables(int nx, int ny, int nxe, int nye, std::vector<double>& h);
// scratch of the coarse-to-fine sweep per batch item (elements of T)
size_t sweep_doubles(int nx, int ny, int L);

// the sweep's edge maps A_x (NI x NI) then A_y (NJ x NJ) in FP64 and FP32, one
// device copy per (device, nx, ny) in the process
struct EdgeMaps {
    double* m64 = nullptr;
    float* m32 = nullptr;
    ~EdgeMaps();
};

struct CosTables {
    double* d64 = nullptr;  // owned device block (nullptr when attached to external memory)
    float* d32 = nullptr;
    std::shared_ptr<struct EdgeMaps> maps;  // edge maps, shared by every context with the same grid size
    GridTables<double> t64;
    GridTables<float> t32;
    int init(int nx, int ny, int nxe, int nye);
    // the sweep's linear map from boundary-line sums to the finer level's boundary
    // DSTs, one matrix per direction, built with the FFT tables (optional)
    int build_edge_maps(int nx, int ny, int nxe, int nye, const FftTables& ft);
    void attach(int nx, int ny, double* p64, float* p32);
    void release();
};

bool fft_supported(int m);
// sin(pi j / N), j = 0 .. N / 2: the half-length DST's pre-processing sines
void fill_dst_sines(int N, double* out);
// Scalar::coarsify of a field in place (every level, finest first)
void coarsify_field(const GridDev& g, double* f, cudaStream_t st);
// the coarsified overlap interiors of levels 1..L-1 of f into rc (f unchanged)
void coarsify_rhs(const GridDev& g, const double* f, double* rc, cudaStream_t st);
// factor m into the radices the shared-memory FFT uses (no device allocation)
void fft_describe(int m, FftDesc& d);

// One multi-domain solve call.  All arrays are device pointers.
template <typename T>
struct SolveCall {
    const T* f;       // right-hand side, all levels
    T* u;             // solution, all levels
    T* rc;            // scratch: coarsified right-hand side (levels 1..L-1), bstride per item;
                      // nullptr: f is already coarsified (its levels are used as they stand)
    T* tbuf;          // scratch: spectral coefficients of all levels (L * N1 per batch item)
    T* sweep;         // scratch: sweep_doubles(nx, ny, L) per batch item
    size_t bstride;   // batch stride of f, u, rc, out2, base
    int batch;
    T in_scale;       // multiplies the right-hand side (+1 or -1)
    T* out2;          // optional: out2 = base - u
    const T* base;
    T* tbuf2 = nullptr;  // scratch of the GEMM passes (L * N1 per batch item; FP32 plans with gemm)
};

template <typename T>
struct EllipticPlan {
    const GridDev* grid = nullptr;
    const FftTables* tables = nullptr;
    const CosTables* cos = nullptr;
    int helmholtz = 0;
    double alpha = 0.0;
    int threads = 128;
    // tuned launch shape of the row and column passes for batch 1 (0: rule-based)
    int rows_P = 0, rows_T = 0, cols_P = 0, cols_T = 0, rows_tws = 0, cols_tws = 0;
    bool edge_maps = true;  // the sweep applies the precomputed edge maps (else the per-step line FFTs)
    // two zeroed device counters owned by the caller: with them (and batch 1) the per-step line FFTs
    // run inside the sums launch, by the last block of each direction; shared by the plans of one stream
    int* sweep_counters = nullptr;
    // the passes' DST form: half-length FFTs (FP64 only) or the odd extension
    bool half = sizeof(T) == 8;
    int set_half(bool h);
    // raises the passes' dynamic shared-memory limits to what rows_P / cols_P line pairs need
    // (at least two pairs); IBG_ERR_UNSUPPORTED when that is above 200 KiB
    int raise_pass_limits() const;
    const FftDesc& pdesc(int pass) const {
        if (half) return pass == 0 ? tables->rowh64 : tables->colh64;
        return sizeof(T) == 8 ? (pass == 0 ? tables->row64 : tables->col64) : (pass == 0 ? tables->row32 : tables->col32);
    }
    const T* psines(int pass) const { return half ? pass_sines<T>(*tables, pass) : nullptr; }
    // FP32 plans: the DST passes as sine-matrix GEMMs on the tensor cores (dst_gemm.cu) instead of FFTs
    bool gemm = false;
    const SineMats* sines = nullptr;
    int solve_gemm(const SolveCall<T>& c, cudaStream_t st) const;
    void run_sweep(const SolveCall<T>& c, const T* coef, cudaStream_t st) const;
    int init(const GridDev* g, const FftTables* t, bool helm, double a, const CosTables& ct);
    int solve(const SolveCall<T>& c, cudaStream_t st) const;
    int launches(bool coarsify = true) const;
    // one pass of the forward transform of all levels alone (0: rows, 1: columns), for timing
    void run_pass(int which, const T* in, T* tbuf, cudaStream_t st) const;
    const GridTables<T>& tabs() const;
    void launch_rows(const GridDev& g, const FftDesc& frow, int nlev, int batch, const T* const* in,
                     const T* const* alt, size_t in_bs, T* const* out, size_t out_bs, T* const* out2,
                     const T* const* base, T scale, T norm, cudaStream_t st) const;
    void launch_cols(const GridDev& g, const FftDesc& fcol, int mode, int nlev, int batch, T* buf, size_t lstride,
                     size_t bstride, const T* edges, size_t estride, cudaStream_t st) const;
};

// autotuner of the row/column passes (elliptic.cu): time the launch shapes once per
// (precision, pass, FFT length, line count, level count) in the process
template <typename T>
int tune_passes(const GridDev* g, const FftTables* t, const CosTables& ct, const SolveCall<T>& call, cudaStream_t st,
                bool half);
void tuned_config(int wbytes, int pass, int m, int nlines, int nlev, int& P, int& nt, int& tws);
struct TuneResult {
    int wbytes, pass, m, nlines, nlev, P, threads, tw_smem;
};
std::vector<TuneResult> tune_log();

// One FP64-accurate solve from FP32 transforms (refine.cu): the FP32 solve of the
// coarsified right-hand side, its FP64 residual on every level, the FP32 solve of
// the residual, and the FP64 sum.  rc64 (S doubles) and f32, u32, d32 (S floats)
// are scratch, tbuf32, tbuf2_32 and sweep32 the FP32 plan's transform scratch; batch 1.
int refined_solve(const GridDev& g, const EllipticPlan<float>& plan32, const SolveCall<double>& c, double* rc64,
                  float* f32, float* u32, float* d32, float* tbuf32, float* tbuf2_32, float* sweep32, cudaStream_t st);
int refined_solve_launches(const GridDev& g, const EllipticPlan<float>& plan32);

template <>
inline const GridTables<double>& EllipticPlan<double>::tabs() const { return cos->t64; }
template <>
inline const GridTables<float>& EllipticPlan<float>::tabs() const { return cos->t32; }

}  // namespace ibg
