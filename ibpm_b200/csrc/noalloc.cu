// noalloc.cu -- a multi-domain Poisson solve that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code running while a CUDA graph is
// being captured into a caller-owned memory pool, plug-ins whose host
// application forbids device allocation after start-up, or services that
// pre-plan every byte of HBM.  For them ibg_poisson_solve_static takes device
// input and output buffers and keeps its scratch (the coarsified right-hand
// side and the transform workspace) in the file-scope array below, plus the
// FFT twiddle and eigenvalue cosine tables of up to kTableSlots grid shapes in
// two more file-scope arrays.  Every GPU that loads the library holds these
// arrays until the process exits.
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ibpm_b200.h"
#include "ibg_internal.cuh"
#include "ibg_kernels.cuh"

using namespace ibg;

namespace {

// 4 MiB of scratch: the coarsified right-hand side, the spectral coefficients
// of every level and the coarse-to-fine sweep workspace must fit in it
constexpr size_t kStaticScratchDoubles = (size_t)1 << 19;
// twiddles for FFT lengths up to 2 * 2048 (nx, ny <= 2048) and the grid tables,
// one block per grid shape for up to kTableSlots shapes
constexpr int kStaticMaxM = 4096;
constexpr int kStaticMaxN = 2048;
// per slot: the row and column twiddles of the sweep's length-2n FFTs, then those
// of the passes' length-n FFTs
constexpr size_t kStaticTwiddles = 2 * (size_t)kStaticMaxM + 2 * (size_t)kStaticMaxN;
// per slot: the grid's cosine and sine tables, then the passes' pre-processing
// sines of the rows (from kSinRow) and the columns (from kSinCol), n / 2 + 1 each
constexpr size_t kSinRow = 10 * (size_t)kStaticMaxN;
constexpr size_t kSinCol = kSinRow + kStaticMaxN / 2 + 8;
constexpr size_t kStaticTableDoubles = kSinCol + kStaticMaxN / 2 + 8;
constexpr int kTableSlots = 4;

static __device__ __align__(256) double g_static_scratch[kStaticScratchDoubles];
static __device__ __align__(256) double2 g_static_twiddles[kTableSlots * kStaticTwiddles];
static __device__ __align__(256) double g_static_cos[kTableSlots * kStaticTableDoubles];

struct TableSlot {
    int nx = -1, ny = -1;        // shape the slot holds (-1: empty)
    unsigned long long used = 0; // last use, for least-recently-used replacement
};
struct DeviceSymbols {
    bool ready = false;
    double* scratch = nullptr;
    double2* twiddles = nullptr;
    double* cosines = nullptr;
    TableSlot slot[kTableSlots];
    unsigned long long clock = 0;
};
constexpr int kMaxDevices = 64;
DeviceSymbols g_dev[kMaxDevices];
std::mutex g_mutex;
// the last failure of the calling thread
thread_local std::string g_static_error;

// doubles of scratch one solve needs: rc (L N1) + coefficients (L N1) + sweep
size_t static_scratch_need(int nx, int ny, int L) {
    const size_t N1 = (size_t)(nx - 1) * (ny - 1);
    return 2 * (size_t)L * N1 + sweep_doubles(nx, ny, L);
}

int fail(int code, const std::string& m) {
    g_static_error = m;
    return code;
}

// writes the twiddles and grid tables of an nx x ny grid into table slot `k`
int fill_slot(DeviceSymbols& ds, int k, int nx, int ny, int nxe, int nye, cudaStream_t st) {
    const double pi = 3.14159265358979323846264338327950288;
    std::vector<double2> tw(kStaticTwiddles);
    auto twiddles = [&](int m, size_t at) {
        for (int j = 0; j < m; ++j) {
            const double a = -2.0 * pi * (double)j / (double)m;
            tw[at + j] = make_double2(cos(a), sin(a));
        }
    };
    twiddles(2 * ny, 0);
    twiddles(2 * nx, kStaticMaxM);
    twiddles(ny, 2 * (size_t)kStaticMaxM);
    twiddles(nx, 2 * (size_t)kStaticMaxM + kStaticMaxN);
    std::vector<double> cs;
    fill_grid_tables(nx, ny, nxe, nye, cs);
    cs.resize(kStaticTableDoubles, 0.0);
    fill_dst_sines(ny, cs.data() + kSinRow);
    fill_dst_sines(nx, cs.data() + kSinCol);
    if (cudaMemcpyAsync(ds.twiddles + (size_t)k * kStaticTwiddles, tw.data(), sizeof(double2) * tw.size(),
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(ds.cosines + (size_t)k * kStaticTableDoubles, cs.data(), sizeof(double) * cs.size(),
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(IBG_ERR_CUDA, "ibg_poisson_solve_static: table upload failed");
    return IBG_OK;
}

}  // namespace

extern "C" const char* ibg_static_last_error(void) { return g_static_error.c_str(); }

extern "C" int ibg_poisson_solve_static(const ibg_grid* grid, const double* f, double* u, void* cuda_stream) {
    if (!grid || !f || !u) return fail(IBG_ERR_ARG, "ibg_poisson_solve_static: null argument");
    const int nx = grid->nx, ny = grid->ny, L = grid->ngrid;
    if (nx < 4 || ny < 4 || L < 1 || L > 16 || !(grid->length > 0))
        return fail(IBG_ERR_ARG, "ibg_poisson_solve_static: invalid grid");
    if (L > 1 && (nx % 2 || ny % 2))
        return fail(IBG_ERR_ARG, "ibg_poisson_solve_static: nx and ny must be even when ngrid > 1");
    if (nx > kStaticMaxN || ny > kStaticMaxN)
        return fail(IBG_ERR_UNSUPPORTED, "ibg_poisson_solve_static: nx and ny must be <= 2048 (static tables)");
    const size_t N1 = (size_t)(nx - 1) * (ny - 1);
    const size_t need = static_scratch_need(nx, ny, L);
    if (need > kStaticScratchDoubles)
        return fail(IBG_ERR_UNSUPPORTED,
                    "ibg_poisson_solve_static: the grid needs " + std::to_string(need) +
                        " doubles of scratch, more than the 524288-double (4 MiB) static scratch; "
                        "use ibg_poisson_solve");
    if (!fft_supported(2 * nx) || !fft_supported(2 * ny) || !fft_supported(nx) || !fft_supported(ny))
        return fail(IBG_ERR_UNSUPPORTED, "ibg_poisson_solve_static: 2*nx and 2*ny must factor into primes <= 13");
    cudaStream_t st = (cudaStream_t)cuda_stream;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(IBG_ERR_CUDA, "ibg_poisson_solve_static: no usable CUDA device");
    const int nxe = (int)floor(nx / 4 + 0.5), nye = (int)floor(ny / 4 + 0.5);

    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceSymbols& ds = g_dev[dev];
    if (!ds.ready) {
        // host-side stand-ins are not device addresses: resolve them once per device
        cudaError_t e1 = cudaGetSymbolAddress((void**)&ds.scratch, g_static_scratch);
        cudaError_t e2 = cudaGetSymbolAddress((void**)&ds.twiddles, g_static_twiddles);
        cudaError_t e3 = cudaGetSymbolAddress((void**)&ds.cosines, g_static_cos);
        cudaError_t e = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3);
        if (e != cudaSuccess)
            return fail(IBG_ERR_CUDA, std::string("ibg_poisson_solve_static: cudaGetSymbolAddress failed: ") +
                                          cudaGetErrorString(e));
        ds.ready = true;
    }
    // the table slot of this shape, or the least recently used one refilled
    int k = -1;
    for (int s = 0; s < kTableSlots; ++s)
        if (ds.slot[s].nx == nx && ds.slot[s].ny == ny) k = s;
    if (k < 0) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
            return fail(IBG_ERR_UNSUPPORTED,
                        "ibg_poisson_solve_static: a grid shape's first call uploads its tables and cannot run while "
                        "the stream is being captured; call once with this shape before capturing");
        k = 0;
        for (int s = 1; s < kTableSlots; ++s)
            if (ds.slot[s].used < ds.slot[k].used) k = s;
        ds.slot[k].nx = -1;
        const int s = fill_slot(ds, k, nx, ny, nxe, nye, st);
        if (s != IBG_OK) return s;
        ds.slot[k].nx = nx;
        ds.slot[k].ny = ny;
    }
    ds.slot[k].used = ++ds.clock;
    double2* twid = ds.twiddles + (size_t)k * kStaticTwiddles;
    double* cosines = ds.cosines + (size_t)k * kStaticTableDoubles;

    GridDev g{};
    g.nx = nx;
    g.ny = ny;
    g.L = L;
    g.nxe = nxe;
    g.nye = nye;
    g.NI = nx - 1;
    g.NJ = ny - 1;
    g.N1 = g.NI * g.NJ;
    g.nXf = (nx + 1) * ny;
    g.F1 = 2 * nx * ny + nx + ny;
    g.dx = grid->length / nx;
    g.x0 = grid->xoffset;
    g.y0 = grid->yoffset;

    FftTables tables;  // descriptors only; twiddles and sines live in the static arrays
    fft_describe(2 * ny, tables.row64);
    fft_describe(2 * nx, tables.col64);
    fft_describe(ny, tables.rowh64);
    fft_describe(nx, tables.colh64);
    tables.row64.tw = twid;
    tables.col64.tw = twid + kStaticMaxM;
    tables.rowh64.tw = twid + 2 * kStaticMaxM;
    tables.colh64.tw = twid + 2 * kStaticMaxM + kStaticMaxN;
    tables.sin_row64 = cosines + kSinRow;
    tables.sin_col64 = cosines + kSinCol;
    CosTables ct;  // views into g_static_cos; owns nothing
    ct.attach(nx, ny, cosines, nullptr);
    EllipticPlan<double> plan;
    const int si = plan.init(&g, &tables, false, 0.0, ct);
    if (si == IBG_ERR_UNSUPPORTED)
        return fail(IBG_ERR_UNSUPPORTED,
                    "ibg_poisson_solve_static: the transform kernels' shared memory for this grid exceeds 200 KiB "
                    "(16*max(2nx,2ny)*2 + 48*max(nx-1,ny-1) bytes); use ibg_poisson_solve");
    if (si != IBG_OK)
        return fail(IBG_ERR_CUDA, "ibg_poisson_solve_static: raising the kernels' shared-memory limit failed");

    SolveCall<double> c{};
    c.f = f;
    c.u = u;
    c.rc = ds.scratch;                        // levels 1..L-1 at rc + lev*N1
    c.tbuf = ds.scratch + (size_t)L * N1;     // spectral coefficients of every level
    c.sweep = ds.scratch + (size_t)2 * L * N1;
    c.bstride = (size_t)L * N1;
    c.batch = 1;
    c.in_scale = 1.0;
    const int s = plan.solve(c, st);
    if (s != IBG_OK || cudaPeekAtLastError() != cudaSuccess)
        return fail(IBG_ERR_CUDA, std::string("ibg_poisson_solve_static: launch failed: ") +
                                      cudaGetErrorString(cudaGetLastError()));
    return IBG_OK;
}
