// api.cu -- the C ABI (include/ibpm_b200.h): context, state, time step.
//
// One context = one IBPM simulation resident in HBM: the reference's
// NavierStokesModel + NonlinearIBSolver + State (src/NavierStokesModel.*,
// src/IBSolver.*, src/State.*).  A time step is a fixed sequence of kernel
// launches on one stream; for fixed bodies the whole step is captured once
// into a CUDA graph and replayed.  Moving bodies use CG, whose convergence
// test is read back every few iterations.
#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdio>
#include <random>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include <array>
#include <map>
#include <mutex>

#include "../../include/ibpm_b200.h"
#include "../../include/ibpm_b200_diag.h"
#include "ibg_force.cuh"
#include "ibg_internal.cuh"
#include "ibg_kernels.cuh"
#include "ibg_lpc.cuh"
#include "ibg_ops.cuh"

using namespace ibg;

namespace {
thread_local std::string g_create_error;

struct Scheme {
    int nsub;
    double an[4], bn[4], cn[4];
};

// coefficients of src/Scheme.h:13-61
Scheme make_scheme(int s) {
    Scheme r{};
    if (s == IBG_SCHEME_EULER) {
        r.nsub = 1;
        r.an[0] = 1.; r.bn[0] = 0.; r.cn[0] = 1.;
    } else if (s == IBG_SCHEME_AB2) {
        r.nsub = 1;
        r.an[0] = 3. / 2.; r.bn[0] = -1. / 2.; r.cn[0] = 1.;
    } else if (s == IBG_SCHEME_RK3) {
        r.nsub = 3;
        r.an[0] = 8. / 15.; r.an[1] = 5. / 12.; r.an[2] = 3. / 4.;
        r.bn[0] = 0.; r.bn[1] = -17. / 60.; r.bn[2] = -5. / 12.;
        r.cn[0] = 8. / 15.; r.cn[1] = 2. / 3.; r.cn[2] = 1.;
    } else if (s == IBG_SCHEME_RK3B) {
        r.nsub = 4;
        r.an[0] = 8. / 17.; r.an[1] = 17. / 60.; r.an[2] = 5. / 12.; r.an[3] = 3. / 4.;
        r.bn[0] = 0.; r.bn[1] = -15. / 68.; r.bn[2] = -17. / 60.; r.bn[3] = -5. / 12.;
        r.cn[0] = 8. / 17.; r.cn[1] = 8. / 15.; r.cn[2] = 2. / 3.; r.cn[3] = 1.;
    } else {
        r.nsub = 0;
    }
    return r;
}

constexpr int kHistCap = 1 << 16;
constexpr int kExtNow = 4;  // external-kinematics slot of "now" (slots 0..3: the sub-steps)
}  // namespace

// bulk fields and solver plans in one arithmetic type
template <typename T>
struct Bulk {
    T *w = nullptr, *q = nullptr, *a = nullptr, *ws = nullptr, *psi = nullptr, *cc = nullptr, *rc = nullptr;
    T *tbuf = nullptr, *sweep = nullptr, *U = nullptr, *V = nullptr, *C = nullptr, *Bf = nullptr, *qtmp = nullptr;
    T* Nbuf[4] = {nullptr, nullptr, nullptr, nullptr};
    T* tbuf2 = nullptr;  // FP32 plans: the GEMM passes' second coefficient buffer
    EllipticPlan<T> poisson;
    EllipticPlan<T> helm[4];
    bool ready = false;
    void release() {
        T* ptrs[] = {w, q, a, ws, psi, cc, rc, tbuf, sweep, U, V, C, Bf, qtmp, Nbuf[0], Nbuf[1], Nbuf[2], Nbuf[3], tbuf2};
        for (T* p : ptrs)
            if (p) cudaFree(p);
        w = q = a = ws = psi = cc = rc = tbuf = sweep = U = V = C = Bf = qtmp = tbuf2 = nullptr;
        for (auto& n : Nbuf) n = nullptr;
        ready = false;
    }
};

namespace ibg {
// End of one device-side CG iteration: keep looping while the solve is active.
// flags: [0] active, [1] iterations of this solve, [2] cap, [3] total iterations,
// [4] solves, [5] largest count, [6] solves that hit the cap, [7] loop counter.
// The loop also stops after cap + 2 passes whatever the solver flags say.
__global__ void k_cg_loop_cond(cudaGraphConditionalHandle h, int* flags) {
    pdl_enter();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int loops = flags[7] + 1;
    flags[7] = loops;
    const bool more = flags[0] != 0 && loops <= flags[2] + 2;
    if (!more) {
        const int it = flags[1];
        flags[3] += it;
        flags[4] += 1;
        if (it > flags[5]) flags[5] = it;
        if (it >= flags[2]) flags[6] += 1;
    }
    cudaGraphSetConditional(h, more ? 1u : 0u);
}
__global__ void k_cg_loop_reset(int* flags) {
    pdl_enter();
    if (threadIdx.x == 0 && blockIdx.x == 0) flags[7] = 0;
}

// one external-kinematics slot ([x.., y..] points then velocities) into the interleaved device layout
__global__ void k_ext_boundary(int npts, const double* __restrict__ ext, double* __restrict__ pts,
                               double* __restrict__ vel) {
    pdl_enter();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npts) return;
    pts[2 * p] = ext[p];
    pts[2 * p + 1] = ext[npts + p];
    vel[2 * p] = ext[2 * npts + p];
    vel[2 * p + 1] = ext[3 * npts + p];
}

__global__ void k_scale(size_t n, const double* __restrict__ in, double s, double* __restrict__ out) {
    pdl_enter();
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = s * in[i];
}

template <typename A, typename B>
__global__ void k_convert(size_t n, const A* __restrict__ in, B* __restrict__ out) {
    pdl_enter();
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (B)in[i];
}
}  // namespace ibg

namespace {
// The autotuner's choice between the FFT and the sine-matrix GEMM form of the FP32
// DST passes, once per grid shape in the process: {nx, ny, levels} -> {gemm chosen,
// FFT us, GEMM us} (median of 5 trials of 8 whole Poisson solves each).
std::mutex g_form_mu;
std::map<std::array<int, 3>, std::array<double, 3>> g_form;

// The autotuner's choice of the FP64 DST passes' form, once per grid shape: {nx, ny, levels} ->
// {half length chosen, half-length us, odd-extension us} per whole Poisson solve.
std::mutex g_pform_mu;
std::map<std::array<int, 3>, std::array<double, 3>> g_pform;

// The autotuner's choice between the coarse-to-fine sweep's edge maps and its per-step line FFTs (fused
// into the sums launch), once per grid shape and precision: {nx, ny, levels, bytes per word} ->
// {edge maps chosen, edge-map us, line-FFT us} per whole Poisson solve.
std::mutex g_sweep_mu;
std::map<std::array<int, 4>, std::array<double, 3>> g_sweep;

template <typename T>
double time_solves(const EllipticPlan<T>& p, const SolveCall<T>& c, cudaStream_t st) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int w = 0; w < 3; ++w) p.solve(c, st);
    std::vector<float> ms;
    for (int t = 0; t < 5; ++t) {
        cudaEventRecord(e0, st);
        for (int r = 0; r < 8; ++r) p.solve(c, st);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float v = 0.f;
        cudaEventElapsedTime(&v, e0, e1);
        ms.push_back(v);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::sort(ms.begin(), ms.end());
    return 1000.0 * ms[2] / 8.0;
}
}  // namespace

struct ibg_context {
    // configuration
    GridDev g{};
    size_t S = 0, F = 0;
    ibg_params prm{};
    Scheme sch{};
    double u0 = 0, v0 = 0;
    int npts = 0, ncomp = 0;
    bool moving = false;
    // external kinematics: the caller moves the bodies (host Geometry) and hands the device the points
    // and velocities of each sub-step; d_ext holds kExtNow + 1 slots of [points | velocities] (2 npts
    // each, BoundaryVector layout)
    bool ext_kin = false;
    double* d_ext = nullptr;
    bool fp32 = false;  // bulk fields of the time step in FP32
    bool refined = false;  // FP64 state, every time-step solve from FP32 transforms + one FP64-residual refinement
    cudaStream_t st = nullptr;
    bool own_stream = false;
    std::string err;
    // plans and bulk fields (FP64 always: state I/O, operator entry points, Cholesky build)
    FftTables fft;
    CosTables cosT;
    Bulk<double> b64;
    Bulk<float> b32;
    SineMats sines;  // FP32 plans: S_x, S_y split for 3xTF32 (dst_gemm.cu)
    // every FP32 plan's DST passes as sine-matrix GEMMs on the tensor cores, or as FFTs
    void set_dst_gemm(bool on) {
        b32.poisson.gemm = on;
        for (int k = 0; k < 4; ++k) b32.helm[k].gemm = on;
        drop_graph();
    }
    // time whole FP32 solves with the FFT and the GEMM passes the first time a grid shape is
    // created in the process; keep the GEMM form if it is at least 3 % faster
    int choose_dst_form() {
        const std::array<int, 3> key = {g.nx, g.ny, g.L};
        {
            std::lock_guard<std::mutex> lock(g_form_mu);
            auto it = g_form.find(key);
            if (it != g_form.end()) {
                set_dst_gemm(it->second[0] > 0.5);
                return IBG_OK;
            }
        }
        SolveCall<float> c = call<float>(b32, b32.a, b32.ws, 1.0f);
        cudaMemsetAsync(b32.a, 0, sizeof(float) * S, st);
        set_dst_gemm(false);
        const double t_fft = time_solves<float>(b32.poisson, c, st);
        set_dst_gemm(true);
        const double t_gemm = time_solves<float>(b32.poisson, c, st);
        int e = 0;
        if (sines.err) {
            cudaMemcpyAsync(&e, sines.err, sizeof(int), cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
        }
        const bool use = e == 0 && t_gemm < 0.97 * t_fft;
        set_dst_gemm(use);
        std::lock_guard<std::mutex> lock(g_form_mu);
        g_form[key] = {use ? 1.0 : 0.0, t_fft, t_gemm};
        return cuda_check("choose_dst_form");
    }
    // time whole FP64 solves with the half-length and with the odd-extension DST passes the first time a
    // grid shape is created in the process; keep the half length unless the odd extension is at least 3 %
    // faster (the half length saves an FFT stage and half the shared memory; its pre- and
    // post-processing, a prefix scan among them, cost more than that saves on short lines)
    int choose_pass_form(Bulk<double>& B) {
        const std::array<int, 3> key = {g.nx, g.ny, g.L};
        auto set = [&](bool h) -> int {
            int e = B.poisson.set_half(h);
            for (int k = 0; k < 4 && !e; ++k)
                if (B.helm[k].grid) e = B.helm[k].set_half(h);
            return e ? fail(IBG_ERR_CUDA, "DST pass form: shared-memory limit") : IBG_OK;
        };
        {
            std::lock_guard<std::mutex> lock(g_pform_mu);
            auto it = g_pform.find(key);
            if (it != g_pform.end()) return set(it->second[0] > 0.5);
        }
        SolveCall<double> c = call<double>(B, B.a, B.ws, 1.0);
        cudaMemsetAsync(B.a, 0, sizeof(double) * S, st);
        int e = set(true);
        if (e) return e;
        const double t_half = time_solves<double>(B.poisson, c, st);
        if ((e = set(false))) return e;
        const double t_odd = time_solves<double>(B.poisson, c, st);
        const bool half = !(t_odd < 0.97 * t_half);
        if ((e = set(half))) return e;
        std::lock_guard<std::mutex> lock(g_pform_mu);
        g_pform[key] = {half ? 1.0 : 0.0, t_half, t_odd};
        return cuda_check("choose_pass_form");
    }
    // time whole solves of plans B with the sweep's edge maps and with its fused line FFTs the first time
    // a grid shape is created in the process (per precision); keep the edge maps unless the line FFTs
    // are at least 3 % faster
    template <typename T>
    int choose_sweep_form(Bulk<T>& B) {
        if (g.L < 2 || !B.poisson.tabs().ax) return IBG_OK;
        const std::array<int, 4> key = {g.nx, g.ny, g.L, (int)sizeof(T)};
        auto set = [&](bool maps) {
            B.poisson.edge_maps = maps;
            for (int k = 0; k < 4; ++k) B.helm[k].edge_maps = maps;
        };
        {
            std::lock_guard<std::mutex> lock(g_sweep_mu);
            auto it = g_sweep.find(key);
            if (it != g_sweep.end()) {
                set(it->second[0] > 0.5);
                return IBG_OK;
            }
        }
        SolveCall<T> c = call<T>(B, B.a, B.ws, (T)1);
        cudaMemsetAsync(B.a, 0, sizeof(T) * S, st);
        set(true);
        const double t_maps = time_solves<T>(B.poisson, c, st);
        set(false);
        const double t_lines = time_solves<T>(B.poisson, c, st);
        const bool maps = !(t_lines < 0.97 * t_maps);
        set(maps);
        std::lock_guard<std::mutex> lock(g_sweep_mu);
        g_sweep[key] = {maps ? 1.0 : 0.0, t_maps, t_lines};
        return cuda_check("choose_sweep_form");
    }
    double beta[4] = {0, 0, 0, 0};
    // bodies
    std::vector<BodyDev> h_bodies;
    std::vector<double> h_ref;
    double *d_ref = nullptr, *d_pts = nullptr, *d_vel = nullptr;
    int* d_body_of = nullptr;
    BodyDev* d_bodies = nullptr;
    // motion history (stateful motions) and the bodies' motion tables
    std::vector<double> h_mtab;
    MotionState* d_mstate = nullptr;
    MotionState* d_mstate_keep = nullptr;
    double* d_mtab = nullptr;
    int nbodies = 0;
    bool stateful = false;
    // moving-frame base flow: the first body's motion carried by the base flow
    bool ubf = false;
    BodyDev* d_bf = nullptr;
    MotionState* d_bf_state = nullptr;
    double* d_bfv = nullptr;   // (xdot', ydot', thetadot') of the flow
    double* d_q0 = nullptr;    // the base flow on every level
    double bf_xc = 0, bf_yc = 0;
    RegSlots slots;
    double* d_b = nullptr;
    double* d_time = nullptr;
    // state (f is FP64 in every form)
    double* f = nullptr;
    int timestep = 0;
    double time = 0;
    bool old_saved = false;
    bool state_in_32 = false;  // the FP32 copy of omega/q is the current one
    // work
    int nring = 0;
    double *flux0 = nullptr, *rhsb = nullptr, *btmp = nullptr;
    int* d_sweep_cnt = nullptr;  // the fused sweep's two counters (EllipticPlan::sweep_counters)
    // Cholesky factors per sub-step
    double* Lr[4] = {nullptr, nullptr, nullptr, nullptr};
    double* Lc[4] = {nullptr, nullptr, nullptr, nullptr};
    double* Ld[4] = {nullptr, nullptr, nullptr, nullptr};
    double* Mi[4] = {nullptr, nullptr, nullptr, nullptr};  // explicit M^-1 = L^-T L^-1 per sub-step
    bool chol_ready = false;
    int* d_status = nullptr;
    // CG
    double *cg_r = nullptr, *cg_d = nullptr, *cg_q = nullptr, *cg_scal = nullptr;
    double *cg_z = nullptr, *cg_zold = nullptr;
    int* cg_flags = nullptr;
    int* h_flags = nullptr;  // pinned
    int cg_last = 0, cg_max = 0, cg_capped = 0;
    long long cg_total = 0, cg_solves = 0;
    int steps_since_pc = 0;
    // learned preconditioner
    Lpc lpc;
    bool lpc_ready = false;
    LpcBodies lb;
    std::vector<int> h_nbr, h_cnt;
    TrainScratch tws;
    // force history
    double* d_hist = nullptr;
    int* d_hist_count = nullptr;
    // the other N(x) forms (src/IBSolver.cc:211-283): 0 nonlinear, 1 linearized (period >= 1), 2 SFD
    int nmode = 0;
    int period = 0;
    double* d_base_w = nullptr;  // period x S base vorticity
    double* d_base_q = nullptr;  // period x F base fluxes
    int* d_ts0 = nullptr;        // State timestep at the last upload (steps since then: d_hist_count)
    double* d_what = nullptr;    // SFD filtered vorticity
    double* d_rprev = nullptr;   // SFD previous filter right-hand side
    double sfd_chi = 0.0, sfd_Delta = 1.0;
    bool sfd_rhs_saved = false;
    // inner-product weights (src/VectorOperations.cc:222-412): [0] Scalar, [1] fine Scalar,
    // [2] Flux, [3] fine Flux; built on first use
    double* d_ipw[4] = {nullptr, nullptr, nullptr, nullptr};
    double* d_ip_tmp = nullptr;  // two operands (F each) and the partial sums
    int build_ip_weights();
    void release_ip() {
        for (double*& p : d_ipw) {
            if (p) cudaFree(p);
            p = nullptr;
        }
        if (d_ip_tmp) cudaFree(d_ip_tmp);
        d_ip_tmp = nullptr;
    }
    void release_variant() {
        double* p[] = {d_base_w, d_base_q, d_what, d_rprev};
        for (double* x : p)
            if (x) cudaFree(x);
        d_base_w = d_base_q = d_what = d_rprev = nullptr;
        nmode = 0;
        period = 0;
    }
    long long hist_steps = 0;
    // graph
    cudaGraph_t graph_def = nullptr;   // the captured step (kept for ensembles)
    cudaGraphExec_t graph = nullptr;
    long long graph_launches = 0;
    long long launches = 0;
    long long last_launches = 0;

    ~ibg_context() { release(); }

    int fail(int code, const std::string& m) {
        err = m;
        return code;
    }
    int cuda_check(const char* where) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return fail(IBG_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
        return IBG_OK;
    }

    template <typename P>
    int alloc(P** p, size_t n, bool zero = true) {
        if (n == 0) n = 1;
        if (cudaMalloc((void**)p, sizeof(P) * n) != cudaSuccess) return fail(IBG_ERR_CUDA, "cudaMalloc failed");
        if (zero) cudaMemset(*p, 0, sizeof(P) * n);
        return IBG_OK;
    }

    template <typename T>
    int alloc_bulk(Bulk<T>& B) {
        int s = alloc(&B.w, S) || alloc(&B.q, F) || alloc(&B.a, S) || alloc(&B.ws, S) || alloc(&B.psi, S) ||
                alloc(&B.cc, S) || alloc(&B.rc, S) || alloc(&B.tbuf, S) ||
                alloc(&B.sweep, sweep_doubles(g.nx, g.ny, g.L)) || alloc(&B.U, S) || alloc(&B.V, S) ||
                alloc(&B.C, F) || alloc(&B.Bf, S) || alloc(&B.qtmp, F);
        for (int k = 0; k < nring && !s; ++k) s = alloc(&B.Nbuf[k], S);
        if (!s && !d_sweep_cnt) s = alloc(&d_sweep_cnt, 2);
        if (!s && std::is_same<T, float>::value) {
            // the sine-matrix GEMM form of the FP32 DST passes (chosen per grid, see set_dst_gemm)
            s = alloc(&B.tbuf2, S) || sines.init(g.nx, g.ny) || gemm_pass_setup();
        }
        if (s) return IBG_ERR_CUDA;
        // time the DST passes' launch shapes for this grid once per process (before the plans read them)
        s = tune_passes<T>(&g, &fft, cosT, call<T>(B, B.a, B.ws, (T)1), st, true);
        if (!s && std::is_same<T, double>::value)  // FP64 passes have the odd-extension form too
            s = tune_passes<T>(&g, &fft, cosT, call<T>(B, B.a, B.ws, (T)1), st, false);
        if (s) return s;
        s = B.poisson.init(&g, &fft, false, 0.0, cosT);
        for (int k = 0; k < sch.nsub && !s; ++k) {
            const double alpha = -beta[k] / 2. * (1. / prm.Re);  // src/ProjectionSolver.cc:33
            s = B.helm[k].init(&g, &fft, true, alpha, cosT);
        }
        if (s) return s;
        // every solve of this context runs on its stream, one after another: one pair of counters
        B.poisson.sweep_counters = d_sweep_cnt;
        for (int k = 0; k < 4; ++k) B.helm[k].sweep_counters = d_sweep_cnt;
        if constexpr (std::is_same<T, float>::value) {
            B.poisson.sines = &sines;
            for (int k = 0; k < 4; ++k) B.helm[k].sines = &sines;
            const char* e = std::getenv("IBG_DST_GEMM");
            if (e && (e[0] == '0' || e[0] == '1')) {
                set_dst_gemm(e[0] == '1');
            } else {
                s = choose_dst_form();
                if (s) return s;
            }
        }
        if constexpr (std::is_same<T, double>::value) {
            s = choose_pass_form(B);
            if (s) return s;
        }
        s = choose_sweep_form<T>(B);
        if (s) return s;
        B.ready = true;
        return IBG_OK;
    }

    // the ensemble members' DST shapes: two line pairs and 128 threads per CTA in every pass, and the
    // per-step line FFTs in every plan (the members' kernels run side by side, where small blocks
    // give more throughput; two pairs per CTA read 16-byte column segments in FP32: 6178 against
    // 5931 member-steps/s with one pair, both in one process)
    void use_rule_shapes() {
        auto reset = [](auto& plan) {
            plan.rows_P = plan.cols_P = 2;
            plan.rows_T = plan.cols_T = 128;
            plan.rows_tws = plan.cols_tws = 0;
            plan.edge_maps = false;
        };
        reset(b64.poisson);
        reset(b32.poisson);
        for (int k = 0; k < 4; ++k) {
            reset(b64.helm[k]);
            reset(b32.helm[k]);
        }
        drop_graph();
    }
    // asynchronous state snapshots (restart output at logger cadence)
    double* snap_dev = nullptr;    // device copy of omega | q | f taken in stream order
    double* snap_host = nullptr;   // pinned host copy
    cudaStream_t snap_st = nullptr;
    cudaEvent_t snap_copied = nullptr, snap_done = nullptr;
    int snap_timestep = -1;
    double snap_time = 0.0;
    bool snap_valid = false;
    void release_snapshot() {
        if (snap_done) cudaEventSynchronize(snap_done);
        if (snap_dev) cudaFree(snap_dev);
        if (snap_host) cudaFreeHost(snap_host);
        if (snap_st) cudaStreamDestroy(snap_st);
        if (snap_copied) cudaEventDestroy(snap_copied);
        if (snap_done) cudaEventDestroy(snap_done);
        snap_dev = snap_host = nullptr;
        snap_st = nullptr;
        snap_copied = snap_done = nullptr;
        snap_valid = false;
    }

    // one launch shape for every DST pass of every plan (pairs 0: the rule); the next step recaptures
    // one launch shape for every plan's DST passes; fails (shape unchanged where refused) when a
    // plan's passes would need more shared memory than a CTA may take
    int set_shapes(int pairs, int threads, bool edge_maps) {
        int st = IBG_OK;
        auto set = [&](auto& plan) {
            const int P0 = plan.rows_P, T0 = plan.rows_T, C0 = plan.cols_P, U0 = plan.cols_T;
            const int rt = plan.rows_tws, ct = plan.cols_tws;
            plan.rows_P = plan.cols_P = pairs;
            plan.rows_T = plan.cols_T = pairs > 0 ? threads : 0;
            plan.rows_tws = plan.cols_tws = 0;
            plan.edge_maps = edge_maps;
            if (!plan.grid) return;
            const int e = plan.raise_pass_limits();
            if (e) {
                plan.rows_P = P0, plan.rows_T = T0, plan.cols_P = C0, plan.cols_T = U0;
                plan.rows_tws = rt, plan.cols_tws = ct;
                if (!st) st = e;
            }
        };
        set(b64.poisson);
        set(b32.poisson);
        for (int k = 0; k < 4; ++k) {
            set(b64.helm[k]);
            set(b32.helm[k]);
        }
        drop_graph();
        return st;
    }

    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        if (graph_def) cudaGraphDestroy(graph_def);
        graph_def = nullptr;
    }
    void release() {
        release_snapshot();
        release_ip();
        release_variant();
        if (d_ts0) cudaFree(d_ts0);
        d_ts0 = nullptr;
        drop_graph();
        b64.release();
        b32.release();
        sines.release();
        release_build_scratch();
        lpc.release();
        tws.release();
        if (lb.start) cudaFree(lb.start);
        if (lb.len) cudaFree(lb.len);
        if (lb.closed) cudaFree(lb.closed);
        lb = LpcBodies{};
        if (d_ext) cudaFree(d_ext);
        d_ext = nullptr;
        void* ptrs[] = {d_ref, d_pts, d_vel, d_body_of, d_bodies, d_mstate, d_mstate_keep, d_mtab, d_bf, d_bf_state, d_bfv, d_q0,
                        slots.idx, slots.w, slots.n, slots.own, slots.contrib, d_b, d_time, f,
                        flux0, rhsb, btmp, d_status, cg_r, cg_d, cg_q, cg_scal, cg_flags, d_hist, d_hist_count, cg_z, cg_zold,
                        d_sweep_cnt};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        for (int k = 0; k < 4; ++k) {
            if (Lr[k]) cudaFree(Lr[k]);
            if (Lc[k]) cudaFree(Lc[k]);
            if (Ld[k]) cudaFree(Ld[k]);
            if (Mi[k]) cudaFree(Mi[k]);
            Lr[k] = Lc[k] = Ld[k] = Mi[k] = nullptr;
        }
        if (h_flags) cudaFreeHost(h_flags);
        h_flags = nullptr;
        fft.release();
        cosT.release();
        if (own_stream && st) cudaStreamDestroy(st);
        st = nullptr;
        if (side) cudaStreamDestroy(side);
        side = nullptr;
        d_ref = d_pts = d_vel = nullptr;
        d_body_of = nullptr;
        d_bodies = nullptr;
        d_mstate = d_mstate_keep = nullptr;
        d_mtab = nullptr;
        d_bf = nullptr;
        d_bf_state = nullptr;
        d_bfv = d_q0 = nullptr;
        slots = RegSlots{};
        d_b = d_time = f = flux0 = rhsb = btmp = nullptr;
        d_status = nullptr;
        cg_r = cg_d = cg_q = cg_scal = cg_z = cg_zold = nullptr;
        cg_flags = nullptr;
        d_hist = nullptr;
        d_hist_count = nullptr;
        d_sweep_cnt = nullptr;
    }

    Bulk<double>& bulk(double*) { return b64; }
    Bulk<float>& bulk(float*) { return b32; }

    // -----------------------------------------------------------------------
    template <typename T>
    SolveCall<T> call(Bulk<T>& B, const T* fin, T* uout, T scale, T* out2 = nullptr, const T* base = nullptr) {
        SolveCall<T> c{};
        c.f = fin;
        c.u = uout;
        c.rc = B.rc;
        c.tbuf = B.tbuf;
        c.sweep = B.sweep;
        c.tbuf2 = B.tbuf2;
        c.bstride = S;
        c.batch = 1;
        c.in_scale = scale;
        c.out2 = out2;
        c.base = base;
        return c;
    }
    long long solve_launches() const {
        return refined ? refined_solve_launches(g, b32.poisson) : b64.poisson.launches();
    }

    // one multi-domain solve of the time step: plan `which` (-1 Poisson, k the sub-step's
    // Helmholtz); FP64 solves of the refined form run as FP32 solves plus one refinement
    template <typename T>
    void esolve(Bulk<T>& B, int which, const SolveCall<T>& c) {
        if constexpr (std::is_same<T, double>::value) {
            if (refined) {
                const EllipticPlan<float>& p32 = which < 0 ? b32.poisson : b32.helm[which];
                refined_solve(g, p32, c, b64.rc, b32.a, b32.ws, b32.cc, b32.tbuf, b32.tbuf2, b32.sweep, st);
                return;
            }
        }
        (which < 0 ? B.poisson : B.helm[which]).solve(c, st);
    }

    // M d = C A^-1 B d  (src/ProjectionSolver.cc:96-101)
    template <typename T>
    void m_apply(Bulk<T>& B, int k, const double* din, double* dout) {
        launch_smear_bf<T>(g, ncomp, slots, din, flux0, B.Bf, beta[k], st);
        esolve<T>(B, k, call<T>(B, B.Bf, B.cc, (T)1));
        esolve<T>(B, -1, call<T>(B, B.cc, B.psi, (T)-1));
        launch_reg_interp<T>(g, ncomp, slots, B.psi, S, 1, nullptr, dout, 0, st);
        launches += 2 + 2 * solve_launches() + 1;
    }

    // CG with warm start x = f (src/ConjugateGradientSolver.cc:35-65); host reads the
    // convergence flag every `chunk` iterations.
    // The CG loop inside a stream capture: prologue, then a WHILE conditional node
    // whose body (one iteration + the loop-condition kernel) is captured on a side
    // stream.  Iteration counts accumulate on the device (flags[3..6]).
    cudaStream_t side = nullptr;
    bool capturing = false;
    template <typename T>
    int cg_solve_graph(Bulk<T>& B, int k, const double* b, double* x) {
        const bool pc = prm.cg_precond != IBG_PRECOND_NONE;
        m_apply<T>(B, k, x, cg_q);
        if (pc) {
            pcg_begin(ncomp, b, cg_q, cg_r, cg_scal, cg_flags, st);
            precondition(k, cg_r, cg_z);
            pcg_begin2(ncomp, cg_r, cg_z, cg_d, cg_scal, cg_flags, st);
        } else {
            cg_begin(ncomp, b, cg_q, cg_r, cg_d, cg_scal, cg_flags, st);
        }
        launch_k(k_cg_loop_reset, 1, 1, 0, st, cg_flags);
        launches += pc ? 3 : 2;
        cudaStreamCaptureStatus cs;
        unsigned long long id = 0;
        cudaGraph_t cgraph = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        if (cudaStreamGetCaptureInfo(st, &cs, &id, &cgraph, &deps, &ndeps) != cudaSuccess ||
            cs != cudaStreamCaptureStatusActive)
            return fail(IBG_ERR_CUDA, "cg graph: stream is not capturing");
        cudaGraphConditionalHandle h;
        if (cudaGraphConditionalHandleCreate(&h, cgraph, 1, cudaGraphCondAssignDefault) != cudaSuccess)
            return cuda_check("cg graph: conditional handle");
        cudaGraphNodeParams p{};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, cgraph, deps, ndeps, &p) != cudaSuccess) return cuda_check("cg graph: while node");
        cudaGraph_t body = p.conditional.phGraph_out[0];
        if (cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
            return cuda_check("cg graph: dependencies");
        if (!side && cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking) != cudaSuccess)
            return cuda_check("cg graph: side stream");
        if (cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
            cudaSuccess)
            return cuda_check("cg graph: body capture");
        cudaStream_t main = st;
        st = side;
        m_apply<T>(B, k, cg_d, cg_q);
        if (pc) {
            pcg_step1(ncomp, x, cg_r, cg_d, cg_q, cg_z, cg_zold, cg_scal, cg_flags, st);
            precondition(k, cg_r, cg_z);
            pcg_step2(ncomp, cg_r, cg_z, cg_zold, cg_d, cg_scal, cg_flags, st);
        } else {
            cg_update(ncomp, x, cg_r, cg_d, cg_q, cg_scal, cg_flags, st);
        }
        launch_k(k_cg_loop_cond, 1, 1, 0, st, h, cg_flags);
        st = main;
        cudaGraph_t out = nullptr;
        if (cudaStreamEndCapture(side, &out) != cudaSuccess) return cuda_check("cg graph: body end");
        return IBG_OK;
    }

    template <typename T>
    int cg_solve(Bulk<T>& B, int k, const double* b, double* x) {
        if (capturing) return cg_solve_graph<T>(B, k, b, x);
        if (prm.cg_precond != IBG_PRECOND_NONE) return pcg_solve<T>(B, k, b, x);
        m_apply<T>(B, k, x, cg_q);
        cg_begin(ncomp, b, cg_q, cg_r, cg_d, cg_scal, cg_flags, st);
        launches += 1;
        int chunk = cg_last > 4 ? cg_last - 2 : 4;
        int done_iters = 0;
        for (;;) {
            for (int c = 0; c < chunk; ++c) {
                m_apply<T>(B, k, cg_d, cg_q);
                cg_update(ncomp, x, cg_r, cg_d, cg_q, cg_scal, cg_flags, st);
                launches += 1;
            }
            done_iters += chunk;
            cudaMemcpyAsync(h_flags, cg_flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) return cuda_check("cg");
            if (h_flags[0] == 0) break;
            if (done_iters > prm.cg_max_iter + chunk) break;
            chunk = 4;
        }
        cg_last = h_flags[1];
        if (cg_last > cg_max) cg_max = cg_last;
        if (cg_last >= prm.cg_max_iter) ++cg_capped;
        cg_total += cg_last;
        ++cg_solves;
        return IBG_OK;
    }

    // z = P r
    void precondition(int k, const double* r, double* z) {
        if (prm.cg_precond == IBG_PRECOND_CHOLESKY) {
            minv_apply(ncomp, Mi[k], r, z, st);
            launches += 1;
        } else {
            apply_learned_precond(k, r, z);
        }
    }
    void apply_learned_precond(int k, const double* r, double* z);

    // flexible preconditioned CG (Polak-Ribiere beta, so a preconditioner that
    // changes between iterations is allowed); same absolute test r.r <= tol^2
    template <typename T>
    int pcg_solve(Bulk<T>& B, int k, const double* b, double* x) {
        m_apply<T>(B, k, x, cg_q);
        pcg_begin(ncomp, b, cg_q, cg_r, cg_scal, cg_flags, st);
        precondition(k, cg_r, cg_z);
        pcg_begin2(ncomp, cg_r, cg_z, cg_d, cg_scal, cg_flags, st);
        launches += 2;
        int chunk = cg_last > 1 ? cg_last : 1;
        int done_iters = 0;
        for (;;) {
            for (int c = 0; c < chunk; ++c) {
                m_apply<T>(B, k, cg_d, cg_q);
                pcg_step1(ncomp, x, cg_r, cg_d, cg_q, cg_z, cg_zold, cg_scal, cg_flags, st);
                precondition(k, cg_r, cg_z);
                pcg_step2(ncomp, cg_r, cg_z, cg_zold, cg_d, cg_scal, cg_flags, st);
                launches += 2;
            }
            done_iters += chunk;
            cudaMemcpyAsync(h_flags, cg_flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) return cuda_check("pcg");
            if (h_flags[0] == 0) break;
            if (done_iters > prm.cg_max_iter + chunk) break;
            chunk = 2;
        }
        cg_last = h_flags[1];
        if (cg_last > cg_max) cg_max = cg_last;
        if (cg_last >= prm.cg_max_iter) ++cg_capped;
        cg_total += cg_last;
        ++cg_solves;
        return IBG_OK;
    }

    // the projection of one sub-step (src/ProjectionSolver.cc:57-79) given a and b
    template <typename T>
    int projection(Bulk<T>& B, int k, const T* a_in, const double* b_in) {
        esolve<T>(B, k, call<T>(B, a_in, B.ws, (T)1));                             // omega* = A^-1 a
        esolve<T>(B, -1, call<T>(B, B.ws, B.psi, (T)-1));                          // psi* = L^-1(-omega*)
        launch_reg_interp<T>(g, ncomp, slots, B.psi, S, 1, b_in, rhsb, 0, st);   // C omega* - b
        launches += 2 * solve_launches() + 1;
        if (!moving) {
            minv_apply(ncomp, Mi[k], rhsb, f, st);                                  // f = M^-1 rhs
            launches += 1;
        } else {
            int s = cg_solve<T>(B, k, rhsb, f);
            if (s) return s;
        }
        launch_smear_bf<T>(g, ncomp, slots, f, flux0, B.Bf, beta[k], st);         // B f
        esolve<T>(B, k, call<T>(B, B.Bf, B.cc, (T)1, B.w, B.ws));                 // omega = omega* - A^-1 B f
        launches += 2 + solve_launches();
        return IBG_OK;
    }

    // q = Curl(L^-1(-omega)) + q0 (src/NavierStokesModel.cc:121-140)
    template <typename T>
    void refresh(Bulk<T>& B) {
        esolve<T>(B, -1, call<T>(B, B.w, B.psi, (T)-1));
        launch_refresh_flux<T>(g, B.psi, B.q, u0, v0, ubf ? d_q0 : nullptr, st);
        launches += solve_launches() + 1;
    }

    // Geometry::moveBodies(time + toff) and Regularizer::update (src/NavierStokesModel.cc:93-99)
    void move_bodies(double toff, int slot = -1) {
        if (ext_kin) {
            // positions and velocities the caller computed (sub-step `slot` of the next step, or now)
            launch_k(k_ext_boundary, (unsigned)((npts + 127) / 128), 128, 0, st, npts,
                     (const double*)(d_ext + (size_t)(slot < 0 ? kExtNow : slot) * 4 * npts), d_pts, d_vel);
            launch_reg_update(g, npts, d_pts, d_vel, slots, d_b, u0, v0, flux0, st);
            launches += 4;
            return;
        }
        if (stateful) {
            launch_motion_state(nbodies, d_bodies, d_time, toff, d_mstate, st);
            launches += 1;
        }
        launch_kinematics(npts, d_ref, d_body_of, d_bodies, d_mstate, d_mtab, d_time, toff, d_pts, d_vel, st);
        launch_reg_update(g, npts, d_pts, d_vel, slots, d_b, u0, v0, flux0, st);
        launches += 4;
    }

    // BaseFlow::moveFlow(time + toff) (src/NavierStokesModel.cc:94) and the constraints it sets
    void frame_flow(double toff) {
        launch_frame_flow(d_bf, d_bf_state, d_mtab, d_time, toff, prm.u_mag, prm.alpha, d_bfv, st);
        launch_frame_flux(g, d_bfv, bf_xc, bf_yc, d_q0, st);
        launch_bcon_field(ncomp, slots, d_vel, d_q0, g.dx, d_b, st);
        launches += 3;
    }

    // IBSolver::advanceSubstep (src/IBSolver.cc:162-198)
    template <typename T>
    int substep(Bulk<T>& B, int k) {
        const double an = sch.an[k], bn = sch.bn[k], cn = sch.cn[k];
        T* Nk;
        T* Np;
        if (sch.nsub == 1) {
            Nk = B.Nbuf[0];
            Np = B.Nbuf[1];
        } else {
            Nk = B.Nbuf[k];
            Np = B.Nbuf[(k + sch.nsub - 1) % sch.nsub];
        }
        bool curl_fused = false;  // the curl of the nonlinear term runs inside the right-hand side's launch
        if constexpr (std::is_same<T, double>::value) {
            if (nmode == 1) {
                launch_nonlinear_lin(g, B.q, B.w, d_base_q, d_base_w, period, d_ts0, d_hist_count, B.U, B.V, B.C,
                                     Nk, st);
            } else if (nmode == 3) {
                // AdjointIBSolver: Laplacian(CrossProduct(q0, q)) - Curl(CrossProduct(q, omega0)); the
                // right-hand-side and omega* buffers are free until later in the sub-step
                launch_flux_cross(g, d_base_q, B.q, B.a, st);
                coarsify_field(g, B.a, st);
                launch_laplacian<T>(g, B.a, B.ws, st);
                launch_nonlinear<T>(g, B.q, d_base_w, B.U, B.V, B.C, Nk, 1, S, F, st);
                launch_sub(S, B.ws, Nk, Nk, st);
                launches += 3 + g.L;
            } else if (nmode == 2) {
                launch_nonlinear<T>(g, B.q, B.w, B.U, B.V, B.C, Nk, 1, S, F, st);
            } else {
                launch_nonlinear_flux<T>(g, B.q, B.w, B.U, B.V, B.C, 1, S, F, st);
                curl_fused = true;
            }
            if (nmode == 2) {
                launch_sfd(S, B.w, d_what, d_rprev, Nk, sfd_chi, sfd_Delta, an, bn, prm.dt, !sfd_rhs_saved, st);
                sfd_rhs_saved = true;
                launches += 1;
            }
        } else {
            launch_nonlinear_flux<T>(g, B.q, B.w, B.U, B.V, B.C, 1, S, F, st);
            curl_fused = true;
        }
        launches += 1 + g.L + (curl_fused ? 0 : 1);
        if (ubf) frame_flow(cn * prm.dt);
        if (moving) move_bodies(cn * prm.dt, k);
        const T* Nprev = nullptr;
        if (bn != 0) Nprev = old_saved ? Np : Nk;
        const double c1 = 0.5 * (1.0 / prm.Re) * (an + bn);
        if (curl_fused)
            launch_curl_rhs<T>(g, B.C, Nk, B.w, Nprev, B.a, c1, an, bn, prm.dt, st);
        else
            launch_rhs<T>(g, B.w, Nk, Nprev, B.a, c1, an, bn, prm.dt, st);
        launches += 1;
        int s = projection<T>(B, k, B.a, d_b);
        if (s) return s;
        refresh<T>(B);
        if (sch.nsub == 1) cudaMemcpyAsync(Np, Nk, sizeof(T) * S, cudaMemcpyDeviceToDevice, st);  // (a copy, not a kernel)
        old_saved = true;
        return IBG_OK;
    }

    int enqueue_step() {
        if (moving && prm.cg_precond == IBG_PRECOND_LEARNED && lpc_ready) {
            // the network's approximate inverse of M at the current body configuration
            lpc.geometry(d_pts, lb, st);
            lpc.operators(sch.nsub, beta, Mi, st);
            launches += 4;
        }
        for (int k = 0; k < sch.nsub; ++k) {
            int s = fp32 ? substep<float>(b32, k) : substep<double>(b64, k);
            if (s) return s;
        }
        add_time(d_time, prm.dt, st);
        net_force_record();
        launches += 2;
        return IBG_OK;
    }

    // make the FP32 copy current (after the FP64 state was written) or the FP64 copy current
    void to32() {
        if (!fp32) return;
        launch_k(k_convert<double, float>, (unsigned)((S + 255) / 256), 256, 0, st, S, b64.w, b32.w);
        launch_k(k_convert<double, float>, (unsigned)((F + 255) / 256), 256, 0, st, F, b64.q, b32.q);
        state_in_32 = true;
    }
    void to64() {
        if (!fp32 || !state_in_32) return;
        launch_k(k_convert<float, double>, (unsigned)((S + 255) / 256), 256, 0, st, S, b32.w, b64.w);
        launch_k(k_convert<float, double>, (unsigned)((F + 255) / 256), 256, 0, st, F, b32.q, b64.q);
    }

    void net_force_record();

    // ---- explicit force operator M = C A^-1 B at the current body configuration
    // (src/CholeskySolver.cc:49-111): columns M e_j for a chunk of j at once
    // (batched solves), Cholesky factor, explicit inverse; one per sub-step.
    double *bs_bf = nullptr, *bs_u = nullptr, *bs_p = nullptr, *bs_rc = nullptr, *bs_tb = nullptr;
    double *bs_fl = nullptr, *bs_sw = nullptr, *bs_M = nullptr;
    size_t bs_chunk = 0;
    void release_build_scratch() {
        double* p[] = {bs_bf, bs_u, bs_p, bs_rc, bs_tb, bs_fl, bs_sw, bs_M};
        for (double* x : p)
            if (x) cudaFree(x);
        bs_bf = bs_u = bs_p = bs_rc = bs_tb = bs_fl = bs_sw = bs_M = nullptr;
        bs_chunk = 0;
    }
    // columns M_k e_j of sub-step k into bs_M (column j at bs_M + j m)
    int build_m(int k) {
        const int m = ncomp;
        const size_t swd = sweep_doubles(g.nx, g.ny, g.L);
        if (!bs_M) {
            // chunk so that the batched scratch stays below ~8 GB
            const size_t per_col = sizeof(double) * (5 * S + (size_t)g.F1 + swd);
            size_t chunk = ((size_t)8 << 30) / per_col;
            if (chunk < 1) chunk = 1;
            if (chunk > (size_t)m) chunk = m;
            if (chunk > 65535) chunk = 65535;
            int s = alloc(&bs_bf, chunk * S) || alloc(&bs_u, chunk * S) || alloc(&bs_p, chunk * S) ||
                    alloc(&bs_rc, chunk * S) || alloc(&bs_tb, chunk * S) || alloc(&bs_fl, chunk * g.F1) ||
                    alloc(&bs_sw, chunk * swd) || alloc(&bs_M, (size_t)m * m, false);
            if (s) {
                release_build_scratch();
                return fail(IBG_ERR_CUDA, "not enough device memory for the force-operator build");
            }
            bs_chunk = chunk;
        }
        const size_t chunk = bs_chunk;
        for (int col0 = 0; col0 < m; col0 += (int)chunk) {
            const int nb = (int)std::min(chunk, (size_t)(m - col0));
            launch_smear_bf_unit<double>(g, m, col0, nb, slots, bs_fl, g.F1, bs_bf, S, beta[k], st);
            SolveCall<double> h{};
            h.f = bs_bf; h.u = bs_u; h.rc = bs_rc; h.tbuf = bs_tb; h.sweep = bs_sw; h.bstride = S;
            h.batch = nb; h.in_scale = 1.0;
            b64.helm[k].solve(h, st);
            SolveCall<double> pc{};
            pc.f = bs_u; pc.u = bs_p; pc.rc = bs_rc; pc.tbuf = bs_tb; pc.sweep = bs_sw; pc.bstride = S;
            pc.batch = nb; pc.in_scale = -1.0;
            b64.poisson.solve(pc, st);
            launch_reg_interp<double>(g, m, slots, bs_p, S, nb, nullptr, bs_M + (size_t)col0 * m, (size_t)m, st);
        }
        return IBG_OK;
    }
    int build_operator() {
        const int m = ncomp;
        for (int k = 0; k < sch.nsub; ++k)
            if (!Lr[k] && (alloc(&Lr[k], (size_t)m * m, false) || alloc(&Lc[k], (size_t)m * m, false) ||
                           alloc(&Ld[k], (size_t)m, false) || alloc(&Mi[k], (size_t)m * m, false)))
                return fail(IBG_ERR_CUDA, "not enough device memory for the Cholesky factors");
        int s = IBG_OK;
        // the moving-body preconditioner: M_k = beta_k C A_k^-1 B differs between sub-steps only
        // through A_k = 1 - beta_k / (2 Re) L, close to 1 at these Reynolds numbers, so one operator
        // (sub-step 0) scaled by beta_0 / beta_k serves every sub-step and the rebuild costs a third
        const bool shared = moving && prm.cg_precond == IBG_PRECOND_CHOLESKY;
        for (int k = 0; k < (shared ? 1 : sch.nsub) && !s; ++k) {
            s = build_m(k);
            if (s) break;
            s = chol_factor(m, bs_M, Lr[k], Lc[k], Ld[k], d_status, st);
            if (!s) chol_inverse(m, Lr[k], Lc[k], Ld[k], Mi[k], st);
            int hs = 0;
            cudaMemcpyAsync(&hs, d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) s = cuda_check("force operator build");
            if (!s && hs) s = fail(IBG_ERR_NUMERIC, "matrix M is not positive definite");
        }
        if (s) return s;
        if (shared)
            for (int k = 1; k < sch.nsub; ++k)
                launch_k(k_scale, (unsigned)(((size_t)m * m + 255) / 256), 256, 0, st, (size_t)m * m,
                         (const double*)Mi[0], beta[0] / beta[k], Mi[k]);
        chol_ready = true;
        return cuda_check("force operator build");
    }

    // capture one whole step (all sub-steps) into a graph, once
    int ensure_graph() {
        if (graph) return IBG_OK;
        cudaGraph_t gr;
        const long long before = launches;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return cuda_check("capture");
        capturing = true;
        int s = enqueue_step();
        capturing = false;
        if (cudaStreamEndCapture(st, &gr) != cudaSuccess || s) {
            launches = before;
            return s ? s : cuda_check("capture end");
        }
        graph_launches = launches - before;
        launches = before;
        if (cudaGraphInstantiate(&graph, gr, 0) != cudaSuccess) {
            cudaGraphDestroy(gr);
            return cuda_check("instantiate");
        }
        graph_def = gr;
        return IBG_OK;
    }
};

namespace ibg {
__global__ void k_hist_force(int npts, const double* f, double dx2, double* hist, int* count) {
    pdl_enter();
    double sx = 0.0, sy = 0.0;
    for (int k = threadIdx.x; k < npts; k += 32) {
        sx += f[k];
        sy += f[npts + k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    if (threadIdx.x == 0) {
        const int i = *count;
        hist[2 * (i % kHistCap)] = sx * dx2;
        hist[2 * (i % kHistCap) + 1] = sy * dx2;
        *count = i + 1;
    }
}
}  // namespace ibg

namespace ibg {
// after a fallback to plain CG (flags[8]), the preconditioner is the identity
__global__ void k_fallback_identity(int m, const int* __restrict__ flags, const double* __restrict__ r,
                                    double* __restrict__ z) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && flags[8]) z[i] = r[i];
}
}  // namespace ibg

void ibg_context::apply_learned_precond(int k, const double* r, double* z) {
    if (lpc_ready) {
        minv_apply(ncomp, Mi[k], r, z, st);
        launch_k(k_fallback_identity, (ncomp + 255) / 256, 256, 0, st, ncomp, cg_flags, r, z);
        launches += 2;
    } else {
        // no network yet: identity (plain CG directions; a copy, not a kernel)
        cudaMemcpyAsync(z, r, sizeof(double) * ncomp, cudaMemcpyDeviceToDevice, st);
    }
}

void ibg_context::net_force_record() {
    launch_k(ibg::k_hist_force, 1, 32, 0, st, npts, f, g.dx * g.dx, d_hist, d_hist_count);
}

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* ibg_last_error(const ibg_context* ctx) {
    if (!ctx) return g_create_error.c_str();
    return ctx->err.c_str();
}

// RigidBody's motion (src/RigidBody.cc:349-493) as device parameters: the
// geometry file's numbers, the PitchPlunge frequencies times 2 pi
// (src/PitchPlunge.h:38-40), the Eldredge family's normalisers maxG computed
// as their constructors do, and the rows of a motion file appended to tab.
// Returns an error message, or nullptr.
static const char* body_motion(const ibg_body& B, double twopi, BodyDev& d, std::vector<double>& tab) {
    static const int nparams[] = {0, 3, 6, 3, 3, 4, 4, 6, 12, 6, 6, 0, 1};
    if (B.motion < IBG_MOTION_NONE || B.motion > IBG_MOTION_FILE_PERIODIC) return "unsupported motion type";
    const int np = nparams[B.motion];
    for (int k = 0; k < np; ++k) {
        if (!std::isfinite(B.params[k])) return "motion parameter is not finite";
        d.p[k] = B.params[k];
    }
    // maxG = G((t2 + t3) / 2) of the ramp (a, t1, t2, t3, t4) (src/EldredgeManeuver.h:42-43);
    // the pitch ramp of EldredgeCombined2 takes `a` in its t4 factor (src/EldredgeCombined2.h:59)
    auto maxG = [](double a, double a4, double t1, double t2, double t3, double t4) {
        const double tt = (t2 + t3) / 2.;
        return log((cosh(a * (tt - t1)) * cosh(a4 * (tt - t4))) / (cosh(a * (tt - t2)) * cosh(a * (tt - t3))));
    };
    switch (B.motion) {
        case IBG_MOTION_PITCHPLUNGE:
            d.p[1] *= twopi;
            d.p[4] *= twopi;
            break;
        case IBG_MOTION_SIGMOIDALSTEP:
            if (d.p[1] == 0) return "sigmoidalstep: DUR must be non-zero";
            break;
        case IBG_MOTION_LAGSTEP1:
        case IBG_MOTION_LAGSTEP2:
            if (d.p[1] == 0 || d.p[2] == 0) return "lagstep: PW and TAU must be non-zero";
            break;
        case IBG_MOTION_ELDREDGE:
        case IBG_MOTION_ELDREDGE1:
        case IBG_MOTION_ELDREDGE2:
            d.p[6] = maxG(d.p[1], d.p[1], d.p[2], d.p[3], d.p[4], d.p[5]);
            if (!std::isfinite(d.p[6]) || d.p[6] == 0) return "eldredge: the ramp's maximum G is zero or not finite";
            break;
        case IBG_MOTION_ELDREDGECOMBINED2:
            d.p[12] = maxG(d.p[1], d.p[1], d.p[2], d.p[3], d.p[4], d.p[5]);
            d.p[13] = maxG(d.p[7], d.p[1], d.p[8], d.p[9], d.p[10], d.p[11]);
            if (!std::isfinite(d.p[12]) || d.p[12] == 0 || !std::isfinite(d.p[13]) || d.p[13] == 0)
                return "eldredgecombined2: a ramp's maximum G is zero or not finite";
            break;
        case IBG_MOTION_FILE_PERIODIC:
            if (d.p[0] == 0) return "motionfileperiodic: period must be non-zero";
            /* fall through */
        case IBG_MOTION_FILE: {
            if (B.table_rows < 0 || (B.table_rows > 0 && !B.table)) return "motion file: missing table";
            for (int r = 0; r < B.table_rows; ++r) {
                for (int k = 0; k < 7; ++k)
                    if (!std::isfinite(B.table[7 * (size_t)r + k])) return "motion file: value is not finite";
                if (r > 0 && B.table[7 * (size_t)r] < B.table[7 * (size_t)(r - 1)])
                    return "motion file: time must increase monotonically";
            }
            d.trows = B.table_rows;
            d.trow0 = (int)(tab.size() / 7);
            tab.insert(tab.end(), B.table, B.table + 7 * (size_t)B.table_rows);
            break;
        }
        default:
            break;
    }
    return nullptr;
}

int ibg_create(const ibg_grid* grid, int nbodies, const ibg_body* bodies, const ibg_params* params,
               void* cuda_stream, ibg_context** out) {
    if (!out || !grid || !params || (nbodies > 0 && !bodies) || nbodies < 1) {
        g_create_error = "ibg_create: null argument or no bodies";
        return IBG_ERR_ARG;
    }
    *out = nullptr;
    const ibg_grid& G = *grid;
    if (G.nx < 4 || G.ny < 4 || G.ngrid < 1 || G.ngrid > 16 || !(G.length > 0)) {
        g_create_error = "ibg_create: invalid grid";
        return IBG_ERR_ARG;
    }
    // the reference asserts multiples of 4 only in debug builds (src/Grid.cc:72); its
    // release build nests with integer division, which the kernels reproduce for even sizes
    if (G.ngrid > 1 && (G.nx % 2 || G.ny % 2)) {
        g_create_error = "ibg_create: nx and ny must be even when ngrid > 1";
        return IBG_ERR_ARG;
    }
    Scheme sch = make_scheme(params->scheme);
    if (sch.nsub == 0) {
        g_create_error = "ibg_create: unknown scheme";
        return IBG_ERR_ARG;
    }
    if (!(params->Re > 0) || !(params->dt > 0)) {
        g_create_error = "ibg_create: Re and dt must be positive";
        return IBG_ERR_ARG;
    }
    if (params->precision != IBG_PRECISION_FP64 && params->precision != IBG_PRECISION_FP32 &&
        params->precision != IBG_PRECISION_FP32_REFINED) {
        g_create_error = "ibg_create: unknown precision";
        return IBG_ERR_ARG;
    }
    if (!fft_supported(2 * G.nx) || !fft_supported(2 * G.ny)) {
        g_create_error = "ibg_create: 2*nx and 2*ny must factor into primes <= 13";
        return IBG_ERR_UNSUPPORTED;
    }
    if (params->device >= 0 && cudaSetDevice(params->device) != cudaSuccess) {
        g_create_error = "ibg_create: cannot select the requested CUDA device";
        return IBG_ERR_CUDA;
    }
    auto* c = new ibg_context();
    c->prm = *params;
    if (c->prm.cg_max_iter <= 0) c->prm.cg_max_iter = 3000;
    if (c->prm.pc_refresh <= 0) c->prm.pc_refresh = 10;
    // a preconditioner that has not converged within a quarter of the iteration cap hands the solve to
    // plain CG, which keeps the other three quarters (at the cap itself no iterations would be left)
    if (c->prm.pc_fallback_iter <= 0) c->prm.pc_fallback_iter = std::max(1, c->prm.cg_max_iter / 4);
    if (c->prm.cg_precond == IBG_PRECOND_LEARNED && c->prm.pc_refresh <= 0) c->prm.pc_refresh = 10;
    if (c->prm.cg_precond < IBG_PRECOND_NONE || c->prm.cg_precond > IBG_PRECOND_LEARNED) {
        delete c;
        g_create_error = "ibg_create: unknown preconditioner";
        return IBG_ERR_ARG;
    }
    if (!(c->prm.cg_tol > 0)) c->prm.cg_tol = 1e-7;
    c->sch = sch;
    GridDev& g = c->g;
    g.nx = G.nx;
    g.ny = G.ny;
    g.L = G.ngrid;
    g.nxe = (int)floor(G.nx / 4 * (1 - 0.0) + 0.5);  // src/Grid.h:60-62 with zero shift
    g.nye = (int)floor(G.ny / 4 * (1 - 0.0) + 0.5);
    g.NI = G.nx - 1;
    g.NJ = G.ny - 1;
    g.N1 = g.NI * g.NJ;
    g.nXf = (G.nx + 1) * G.ny;
    g.F1 = 2 * G.nx * G.ny + G.nx + G.ny;
    g.dx = G.length / G.nx;
    g.x0 = G.xoffset;
    g.y0 = G.yoffset;
    c->S = (size_t)g.L * g.N1;
    c->F = (size_t)g.L * g.F1;
    c->u0 = c->prm.u_mag * cos(c->prm.alpha);
    c->v0 = c->prm.u_mag * sin(c->prm.alpha);
    // bodies
    const double twopi = 8. * atan(1.);
    std::vector<int> body_of;
    for (int b = 0; b < nbodies; ++b) {
        const ibg_body& B = bodies[b];
        if (B.npoints < 1 || !B.xy) {
            delete c;
            g_create_error = "ibg_create: body without points";
            return IBG_ERR_ARG;
        }
        BodyDev d{};
        d.xc = B.xcenter;
        d.yc = B.ycenter;
        d.motion = B.motion;
        const char* merr = body_motion(B, twopi, d, c->h_mtab);
        if (merr) {
            delete c;
            g_create_error = std::string("ibg_create: ") + merr;
            return B.motion < IBG_MOTION_NONE || B.motion > IBG_MOTION_FILE_PERIODIC ? IBG_ERR_UNSUPPORTED : IBG_ERR_ARG;
        }
        if (B.motion != IBG_MOTION_NONE && B.motion != IBG_MOTION_FIXED) c->moving = true;
        if (motion_is_stateful(B.motion)) c->stateful = true;
        c->h_bodies.push_back(d);
        for (int p = 0; p < B.npoints; ++p) {
            c->h_ref.push_back(B.xy[2 * p]);
            c->h_ref.push_back(B.xy[2 * p + 1]);
            body_of.push_back(b);
        }
    }
    c->npts = (int)body_of.size();
    c->ncomp = 2 * c->npts;
    // boundary neighbours (i +- 1..4 along each body, wrapping on closed curves) for the learned preconditioner
    std::vector<int> bstart, blen, bclosed;
    {
        int p0 = 0;
        for (int b = 0; b < nbodies; ++b) {
            const int n = bodies[b].npoints;
            bstart.push_back(p0);
            blen.push_back(n);
            // closed if the end points are about one spacing apart
            std::vector<double> d;
            for (int q = 0; q + 1 < n; ++q)
                d.push_back(std::hypot(bodies[b].xy[2 * q + 2] - bodies[b].xy[2 * q], bodies[b].xy[2 * q + 3] - bodies[b].xy[2 * q + 1]));
            std::sort(d.begin(), d.end());
            const double med = d.empty() ? 0.0 : d[d.size() / 2];
            const double gap = n > 1 ? std::hypot(bodies[b].xy[2 * (n - 1)] - bodies[b].xy[0], bodies[b].xy[2 * (n - 1) + 1] - bodies[b].xy[1]) : 0.0;
            const int closed = (n > 2 && gap < 1.5 * med) ? 1 : 0;
            bclosed.push_back(closed);
            for (int q = 0; q < n; ++q) {
                int cntq = 0;
                for (int off = 1; off <= 4; ++off)
                    for (int sgn = -1; sgn <= 1; sgn += 2) {
                        int j = q + sgn * off;
                        if (closed) j = ((j % n) + n) % n;
                        else if (j < 0 || j >= n) continue;
                        if (j == q) continue;
                        c->h_nbr.push_back(p0 + j);
                        ++cntq;
                    }
                for (int f = cntq; f < 8; ++f) c->h_nbr.push_back(-1);
                c->h_cnt.push_back(cntq);
            }
            p0 += n;
        }
    }
    if (c->ncomp > 16384) {
        delete c;
        g_create_error = "ibg_create: too many boundary points";
        return IBG_ERR_UNSUPPORTED;
    }
    // stream
    if (cuda_stream) {
        c->st = (cudaStream_t)cuda_stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            g_create_error = "ibg_create: no CUDA device or stream creation failed";
            return IBG_ERR_CUDA;
        }
        c->own_stream = true;
    }
    int s = IBG_OK;
    const size_t m = c->ncomp;
    if ((s = c->fft.init(2 * g.ny, 2 * g.nx)) || (s = c->cosT.init(g.nx, g.ny, g.nxe, g.nye)) ||
        (g.L > 1 && (s = c->cosT.build_edge_maps(g.nx, g.ny, g.nxe, g.nye, c->fft)))) {
        g_create_error = "ibg_create: FFT table setup failed";
        delete c;
        return s;
    }
    for (int k = 0; k < sch.nsub; ++k) c->beta[k] = (sch.an[k] + sch.bn[k]) * c->prm.dt;  // src/IBSolver.cc:110-114
    c->nring = sch.nsub == 1 ? 2 : sch.nsub;
    c->fp32 = (c->prm.precision == IBG_PRECISION_FP32);
    c->refined = (c->prm.precision == IBG_PRECISION_FP32_REFINED);
    s = c->alloc_bulk(c->b64);
    if (!s && (c->fp32 || c->refined)) s = c->alloc_bulk(c->b32);
    if (s) {
        g_create_error = "ibg_create: solver set-up or device allocation failed";
        delete c;
        return s;
    }
    s = s || c->alloc(&c->f, m) || c->alloc(&c->flux0, (size_t)g.F1) || c->alloc(&c->rhsb, m) ||
        c->alloc(&c->btmp, m) || c->alloc(&c->d_ref, 2 * (size_t)c->npts) ||
        c->alloc(&c->d_pts, 2 * (size_t)c->npts) || c->alloc(&c->d_vel, 2 * (size_t)c->npts) ||
        c->alloc(&c->d_body_of, (size_t)c->npts) || c->alloc(&c->d_bodies, c->h_bodies.size()) ||
        c->alloc(&c->d_mstate, c->h_bodies.size()) || c->alloc(&c->d_mstate_keep, c->h_bodies.size()) ||
        c->alloc(&c->d_mtab, std::max<size_t>(c->h_mtab.size(), 7)) ||
        c->alloc(&c->slots.idx, kSlots * m) || c->alloc(&c->slots.w, kSlots * m) || c->alloc(&c->slots.n, m) ||
        c->alloc(&c->slots.own, kSlots * m) || c->alloc(&c->slots.contrib, kSlots * m * kMaxContrib) ||
        c->alloc(&c->d_b, m) || c->alloc(&c->d_time, 1) || c->alloc(&c->d_status, 1) || c->alloc(&c->cg_r, m) ||
        c->alloc(&c->cg_d, m) || c->alloc(&c->cg_q, m) || c->alloc(&c->cg_z, m) || c->alloc(&c->cg_zold, m) || c->alloc(&c->cg_scal, 4) || c->alloc(&c->cg_flags, 10) ||
        c->alloc(&c->d_hist, 2 * (size_t)kHistCap) || c->alloc(&c->d_hist_count, 1) || c->alloc(&c->d_ts0, 1);
    if (!s && cudaMallocHost((void**)&c->h_flags, 4 * sizeof(int)) != cudaSuccess) s = IBG_ERR_CUDA;
    if (s) {
        g_create_error = "ibg_create: device allocation failed";
        delete c;
        return IBG_ERR_CUDA;
    }
    cudaMemcpy(c->d_ref, c->h_ref.data(), sizeof(double) * c->h_ref.size(), cudaMemcpyHostToDevice);
    c->slots.pts = c->d_pts;
    c->lb.n = nbodies;
    c->lb.body_of = c->d_body_of;
    if (c->alloc(&c->lb.start, nbodies) || c->alloc(&c->lb.len, nbodies) || c->alloc(&c->lb.closed, nbodies)) {
        g_create_error = "ibg_create: device allocation failed";
        delete c;
        return IBG_ERR_CUDA;
    }
    cudaMemcpy(c->lb.start, bstart.data(), sizeof(int) * nbodies, cudaMemcpyHostToDevice);
    cudaMemcpy(c->lb.len, blen.data(), sizeof(int) * nbodies, cudaMemcpyHostToDevice);
    cudaMemcpy(c->lb.closed, bclosed.data(), sizeof(int) * nbodies, cudaMemcpyHostToDevice);
    cudaMemcpy(c->d_body_of, body_of.data(), sizeof(int) * body_of.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(c->d_bodies, c->h_bodies.data(), sizeof(BodyDev) * c->h_bodies.size(), cudaMemcpyHostToDevice);
    c->nbodies = (int)c->h_bodies.size();
    cudaMemset(c->d_mstate, 0, sizeof(MotionState) * c->h_bodies.size());  // fresh Motion objects: zero history
    if (!c->h_mtab.empty())
        cudaMemcpy(c->d_mtab, c->h_mtab.data(), sizeof(double) * c->h_mtab.size(), cudaMemcpyHostToDevice);
    double sc[4] = {0, 0, c->prm.cg_tol * c->prm.cg_tol, 0};
    cudaMemcpy(c->cg_scal, sc, sizeof(sc), cudaMemcpyHostToDevice);
    int fl[10] = {0, 0, c->prm.cg_max_iter, 0, 0, 0, 0, 0, 0, c->prm.pc_fallback_iter};
    cudaMemcpy(c->cg_flags, fl, sizeof(fl), cudaMemcpyHostToDevice);
    if (chol_solve_prepare((int)m)) {
        g_create_error = "ibg_create: too many boundary points for the Cholesky solve";
        delete c;
        return IBG_ERR_UNSUPPORTED;
    }
    // geom.moveBodies(t = 0); model->init() -> regularizer update
    c->move_bodies(0.0);
    if (cudaStreamSynchronize(c->st) != cudaSuccess || c->cuda_check("ibg_create")) {
        g_create_error = "ibg_create: " + c->err;
        delete c;
        return IBG_ERR_CUDA;
    }
    *out = c;
    return IBG_OK;
}

int ibg_destroy(ibg_context* ctx) {
    if (!ctx) return IBG_ERR_ARG;
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    delete ctx;
    return IBG_OK;
}

// Cholesky build: columns M e_j for a chunk of j at once (batched solves).
int ibg_init(ibg_context* c) {
    if (!c) return IBG_ERR_ARG;
    if (c->moving) {
        if (c->prm.cg_precond == IBG_PRECOND_CHOLESKY) return c->build_operator();
        return IBG_OK;
    }
    if (c->chol_ready) return IBG_OK;
    int s = c->build_operator();
    if (s) return s;
    c->release_build_scratch();
    return IBG_OK;
}

int ibg_save(ibg_context* c, const char* basename) {
    if (!c || !basename) return IBG_ERR_ARG;
    if (c->moving) return 0;  // ProjectionSolver::save returns false for CG
    if (!c->chol_ready) return c->fail(IBG_ERR_STATE, "ibg_save: call ibg_init first");
    const int m = c->ncomp;
    std::vector<double> Lr((size_t)m * m), d(m);
    for (int k = 0; k < c->sch.nsub; ++k) {
        cudaMemcpy(Lr.data(), c->Lr[k], sizeof(double) * m * m, cudaMemcpyDeviceToHost);
        cudaMemcpy(d.data(), c->Ld[k], sizeof(double) * m, cudaMemcpyDeviceToHost);
        char num[16];
        snprintf(num, sizeof(num), "%02d", k + 1);
        std::string fn = std::string(basename) + "_" + num + ".cholesky";
        FILE* fp = fopen(fn.c_str(), "w");
        if (!fp) return c->fail(IBG_ERR_IO, "ibg_save: cannot open " + fn);
        fprintf(fp, "%d\n%.17g\n", m, (1.0 / c->prm.Re) * c->beta[k]);
        for (int i = 0; i < m; ++i) fprintf(fp, "%.17g\n", d[i]);
        fprintf(fp, "#\n");
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < i; ++j) fprintf(fp, "%.17g\n", Lr[(size_t)i * m + j]);
        fclose(fp);
    }
    return 1;
}

int ibg_load(ibg_context* c, const char* basename) {
    if (!c || !basename) return IBG_ERR_ARG;
    if (c->moving) return 0;
    const int m = c->ncomp;
    std::vector<std::vector<double>> Ls(c->sch.nsub), Ds(c->sch.nsub);
    for (int k = 0; k < c->sch.nsub; ++k) {
        char num[16];
        snprintf(num, sizeof(num), "%02d", k + 1);
        std::string fn = std::string(basename) + "_" + num + ".cholesky";
        std::ifstream in(fn.c_str());
        if (!in.good()) return 0;
        int n;
        double ab;
        in >> n;
        if (!in || n != m) return 0;
        in >> ab;
        if (!in || ab != (1.0 / c->prm.Re) * c->beta[k]) return 0;
        Ds[k].resize(m);
        for (int i = 0; i < m; ++i) in >> Ds[k][i];
        char mark = 0;
        in >> mark;
        if (mark != '#') return 0;
        Ls[k].assign((size_t)m * m, 0.0);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < i; ++j) in >> Ls[k][(size_t)i * m + j];
        if (!in) return 0;
    }
    for (int k = 0; k < c->sch.nsub; ++k) {
        if (!c->Lr[k] && (c->alloc(&c->Lr[k], (size_t)m * m) || c->alloc(&c->Lc[k], (size_t)m * m) ||
                          c->alloc(&c->Ld[k], (size_t)m) || c->alloc(&c->Mi[k], (size_t)m * m)))
            return IBG_ERR_CUDA;
        std::vector<double> Lc((size_t)m * m, 0.0);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < i; ++j) Lc[(size_t)j * m + i] = Ls[k][(size_t)i * m + j];
        cudaMemcpy(c->Lr[k], Ls[k].data(), sizeof(double) * m * m, cudaMemcpyHostToDevice);
        cudaMemcpy(c->Lc[k], Lc.data(), sizeof(double) * m * m, cudaMemcpyHostToDevice);
        cudaMemcpy(c->Ld[k], Ds[k].data(), sizeof(double) * m, cudaMemcpyHostToDevice);
        chol_inverse(m, c->Lr[k], c->Lc[k], c->Ld[k], c->Mi[k], c->st);
    }
    cudaStreamSynchronize(c->st);
    c->chol_ready = true;
    return c->cuda_check("ibg_load") ? IBG_ERR_CUDA : 1;
}

// ---------------------------------------------------------------------------
// restart files: State::save / State::load (src/State.cc:65-223).  Layout:
// int nx, ny, ngrid; double dx, x0, y0; int numPoints; q (ngrid x fluxes, the
// Flux index order); omega (ngrid x (nx-1) x (ny-1), j fastest); f as
// (fx, fy) pairs per point; int timestep; double time.  Native byte order.
// ---------------------------------------------------------------------------
static int write_restart(ibg_context* c, const char* filename, const double* w, const double* q, const double* f,
                         int timestep, double time) {
    FILE* fp = fopen(filename, "wb");
    if (!fp) return 0;
    const int hdr_i[3] = {c->g.nx, c->g.ny, c->g.L};
    const double hdr_d[3] = {c->g.dx, c->g.x0, c->g.y0};
    const int np = c->npts;
    bool ok = fwrite(hdr_i, sizeof(int), 3, fp) == 3 && fwrite(hdr_d, sizeof(double), 3, fp) == 3 &&
              fwrite(&np, sizeof(int), 1, fp) == 1 && fwrite(q, sizeof(double), c->F, fp) == c->F &&
              fwrite(w, sizeof(double), c->S, fp) == c->S;
    for (int i = 0; i < np && ok; ++i) {
        const double xy[2] = {f[i], f[np + i]};
        ok = fwrite(xy, sizeof(double), 2, fp) == 2;
    }
    ok = ok && fwrite(&timestep, sizeof(int), 1, fp) == 1 && fwrite(&time, sizeof(double), 1, fp) == 1;
    ok = (fclose(fp) == 0) && ok;
    return ok ? 1 : c->fail(IBG_ERR_IO, std::string("restart file ") + filename + ": write failed");
}

int ibg_save_restart(ibg_context* c, const char* filename) {
    if (!c || !filename) return IBG_ERR_ARG;
    std::vector<double> w(c->S), q(c->F), f(c->ncomp);
    int ts = 0;
    double t = 0.0;
    int s = ibg_get_state(c, w.data(), q.data(), f.data(), &ts, &t);
    if (s) return s;
    return write_restart(c, filename, w.data(), q.data(), f.data(), ts, t);
}

int ibg_load_restart(ibg_context* c, const char* filename) {
    if (!c || !filename) return IBG_ERR_ARG;
    FILE* fp = fopen(filename, "rb");
    if (!fp) return 0;
    int hdr_i[3] = {0, 0, 0}, np = 0, ts = 0;
    double hdr_d[3] = {0, 0, 0}, t = 0.0;
    bool ok = fread(hdr_i, sizeof(int), 3, fp) == 3 && fread(hdr_d, sizeof(double), 3, fp) == 3 &&
              fread(&np, sizeof(int), 1, fp) == 1;
    // the reference resizes its State on a mismatch; a context's grid is fixed, so refuse instead
    if (ok && (hdr_i[0] != c->g.nx || hdr_i[1] != c->g.ny || hdr_i[2] != c->g.L || hdr_d[0] != c->g.dx ||
               hdr_d[1] != c->g.x0 || hdr_d[2] != c->g.y0 || np != c->npts)) {
        fclose(fp);
        return c->fail(IBG_ERR_ARG, std::string("restart file ") + filename +
                                        ": grid or number of boundary points differs from the context's");
    }
    std::vector<double> w(c->S), q(c->F), f(c->ncomp), xy(2 * (size_t)np);
    ok = ok && fread(q.data(), sizeof(double), c->F, fp) == c->F && fread(w.data(), sizeof(double), c->S, fp) == c->S &&
         fread(xy.data(), sizeof(double), xy.size(), fp) == xy.size() && fread(&ts, sizeof(int), 1, fp) == 1 &&
         fread(&t, sizeof(double), 1, fp) == 1;
    fclose(fp);
    if (!ok) return c->fail(IBG_ERR_IO, std::string("restart file ") + filename + ": truncated");
    for (int i = 0; i < np; ++i) {
        f[i] = xy[2 * (size_t)i];
        f[np + i] = xy[2 * (size_t)i + 1];
    }
    int s = ibg_set_state(c, w.data(), q.data(), f.data(), ts, t);
    return s ? s : 1;
}

int ibg_snapshot(ibg_context* c) {
    if (!c) return IBG_ERR_ARG;
    const size_t n = c->S + c->F + c->ncomp;
    if (!c->snap_dev) {
        if (cudaMalloc(&c->snap_dev, sizeof(double) * n) != cudaSuccess ||
            cudaHostAlloc(&c->snap_host, sizeof(double) * n, cudaHostAllocDefault) != cudaSuccess ||
            cudaStreamCreateWithFlags(&c->snap_st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->snap_copied, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->snap_done, cudaEventDisableTiming) != cudaSuccess) {
            c->release_snapshot();
            return c->fail(IBG_ERR_CUDA, "ibg_snapshot: staging set-up failed");
        }
    } else {
        // the previous snapshot's host copy must finish before its device copy is overwritten
        cudaStreamWaitEvent(c->st, c->snap_done, 0);
    }
    c->to64();
    // device copy in stream order (the next steps may run while it travels to the host)
    cudaMemcpyAsync(c->snap_dev, c->b64.w, sizeof(double) * c->S, cudaMemcpyDeviceToDevice, c->st);
    cudaMemcpyAsync(c->snap_dev + c->S, c->b64.q, sizeof(double) * c->F, cudaMemcpyDeviceToDevice, c->st);
    cudaMemcpyAsync(c->snap_dev + c->S + c->F, c->f, sizeof(double) * c->ncomp, cudaMemcpyDeviceToDevice, c->st);
    cudaEventRecord(c->snap_copied, c->st);
    cudaStreamWaitEvent(c->snap_st, c->snap_copied, 0);
    cudaMemcpyAsync(c->snap_host, c->snap_dev, sizeof(double) * n, cudaMemcpyDeviceToHost, c->snap_st);
    cudaEventRecord(c->snap_done, c->snap_st);
    c->snap_timestep = c->timestep;
    c->snap_time = c->time;
    c->snap_valid = true;
    return c->cuda_check("ibg_snapshot");
}

int ibg_snapshot_save(ibg_context* c, const char* filename) {
    if (!c || !filename) return IBG_ERR_ARG;
    if (!c->snap_valid) return c->fail(IBG_ERR_STATE, "ibg_snapshot_save: no snapshot taken");
    if (cudaEventSynchronize(c->snap_done) != cudaSuccess) return c->cuda_check("ibg_snapshot_save");
    const double* h = c->snap_host;
    return write_restart(c, filename, h, h + c->S, h + c->S + c->F, c->snap_timestep, c->snap_time);
}

// ---------------------------------------------------------------------------
// the other N(x) forms
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// inner products and energy (src/VectorOperations.cc:222-412, src/OutputEnergy.cc:29-33)
// ---------------------------------------------------------------------------
namespace ibg {
constexpr int kIpBlocks = 256;
// partial[b] = sum over this block's grid-stride share of w a b (fixed order)
__global__ void k_wdot_partial(size_t n, const double* __restrict__ w, const double* __restrict__ a,
                               const double* __restrict__ b, double* __restrict__ partial) {
    pdl_enter();
    __shared__ double red[32];
    double s = 0.0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        s += w[t] * a[t] * b[t];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
        partial[blockIdx.x] = t;
    }
}
__global__ void k_sum_partials(int n, const double* __restrict__ partial, double scale, double* __restrict__ out) {
    pdl_enter();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < n; ++k) t += partial[k];
        *out = t * scale;
    }
}
}  // namespace ibg

int ibg_context::build_ip_weights() {
    if (d_ipw[0]) return IBG_OK;
    const int nx = g.nx, ny = g.ny, nx2 = g.nxe, ny2 = g.nye, L = g.L;
    const int NI = g.NI, NJ = g.NJ, nXf = g.nXf;
    std::vector<double> ws(S, 0.0), wsf(S, 0.0), wf(F, 0.0), wff(F, 0.0);
    auto sw = [&](std::vector<double>& w, int lev, int i, int j, double v) {
        w[(size_t)lev * g.N1 + (size_t)(i - 1) * NJ + (j - 1)] += v;
    };
    for (int i = 1; i <= NI; ++i)
        for (int j = 1; j <= NJ; ++j) {
            sw(ws, 0, i, j, 1.0);
            sw(wsf, 0, i, j, 1.0);
        }
    for (int lev = 1; lev < L; ++lev) {
        const int il = nx2, ir = nx / 2 + nx2, jb = ny2, jt = ny / 2 + ny2;
        sw(ws, lev, il, jb, 15. / 16); sw(ws, lev, ir, jb, 15. / 16); sw(ws, lev, il, jt, 15. / 16); sw(ws, lev, ir, jt, 15. / 16);
        for (int j = jb + 1; j < jt; ++j) { sw(ws, lev, il, j, 0.75); sw(ws, lev, ir, j, 0.75); }
        for (int i = il + 1; i < ir; ++i) { sw(ws, lev, i, jb, 0.75); sw(ws, lev, i, jt, 0.75); }
        for (int i = 1; i < il; ++i) for (int j = 1; j < ny; ++j) sw(ws, lev, i, j, 1.0);
        for (int i = ir + 1; i < nx; ++i) for (int j = 1; j < ny; ++j) sw(ws, lev, i, j, 1.0);
        for (int i = il; i <= ir; ++i) {
            for (int j = 1; j < jb; ++j) sw(ws, lev, i, j, 1.0);
            for (int j = jt + 1; j < ny; ++j) sw(ws, lev, i, j, 1.0);
        }
    }
    for (int lev = 0; lev < L; ++lev) {
        const double d = lev_dx(g, lev), d2 = d * d;
        for (size_t k = 0; k < (size_t)g.N1; ++k) {
            ws[(size_t)lev * g.N1 + k] *= d2;
            wsf[(size_t)lev * g.N1 + k] *= d2;
        }
    }
    auto xw = [&](std::vector<double>& w, int lev, int i, int j, double v) { w[(size_t)lev * g.F1 + (size_t)i * ny + j] += v; };
    auto yw = [&](std::vector<double>& w, int lev, int i, int j, double v) {
        w[(size_t)lev * g.F1 + nXf + (size_t)i * (ny + 1) + j] += v;
    };
    for (int j = 0; j < ny; ++j) for (int i = 1; i < nx; ++i) { xw(wf, 0, i, j, 1.0); xw(wff, 0, i, j, 1.0); }
    for (int i = 0; i < nx; ++i) for (int j = 1; j < ny; ++j) { yw(wf, 0, i, j, 1.0); yw(wff, 0, i, j, 1.0); }
    for (int lev = 1; lev < L; ++lev) {
        const int il = nx2, ir = nx / 2 + nx2, jb = ny2, jt = ny / 2 + ny2;
        for (int j = jb; j < jt; ++j) { xw(wf, lev, il, j, 0.75); xw(wf, lev, ir, j, 0.75); }
        for (int j = 0; j < ny; ++j) {
            for (int i = 1; i < il; ++i) xw(wf, lev, i, j, 1.0);
            for (int i = ir + 1; i < nx; ++i) xw(wf, lev, i, j, 1.0);
        }
        for (int i = il; i <= ir; ++i) {
            for (int j = 0; j < jb; ++j) xw(wf, lev, i, j, 1.0);
            for (int j = jt; j < ny; ++j) xw(wf, lev, i, j, 1.0);
        }
        for (int i = il; i < ir; ++i) { yw(wf, lev, i, jb, 0.75); yw(wf, lev, i, jt, 0.75); }
        for (int i = 0; i < nx; ++i) {
            for (int j = 1; j < jb; ++j) yw(wf, lev, i, j, 1.0);
            for (int j = jt + 1; j < ny; ++j) yw(wf, lev, i, j, 1.0);
        }
        for (int j = jb; j <= jt; ++j) {
            for (int i = 0; i < il; ++i) yw(wf, lev, i, j, 1.0);
            for (int i = ir; i < nx; ++i) yw(wf, lev, i, j, 1.0);
        }
    }
    const std::vector<double>* src[4] = {&ws, &wsf, &wf, &wff};
    for (int k = 0; k < 4; ++k) {
        if (alloc(&d_ipw[k], src[k]->size(), false)) return IBG_ERR_CUDA;
        cudaMemcpy(d_ipw[k], src[k]->data(), sizeof(double) * src[k]->size(), cudaMemcpyHostToDevice);
    }
    if (alloc(&d_ip_tmp, 2 * (size_t)F + kIpBlocks + 1, false)) return IBG_ERR_CUDA;
    return cuda_check("inner-product weights");
}

static int device_ip(ibg_context* c, int kind, const double* da, const double* db, double scale, double* out) {
    const size_t n = kind < 2 ? c->S : c->F;
    double* partial = c->d_ip_tmp + 2 * (size_t)c->F;
    launch_k(ibg::k_wdot_partial, ibg::kIpBlocks, 256, 0, c->st, n, c->d_ipw[kind], da, db, partial);
    launch_k(ibg::k_sum_partials, 1, 32, 0, c->st, ibg::kIpBlocks, partial, scale, partial + ibg::kIpBlocks);
    cudaMemcpyAsync(out, partial + ibg::kIpBlocks, sizeof(double), cudaMemcpyDeviceToHost, c->st);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("inner product");
    return c->cuda_check("inner product");
}

int ibg_inner_product(ibg_context* c, int kind, const double* a, const double* b, double* ip) {
    if (!c || kind < 0 || kind > 3 || !a || !b || !ip) return IBG_ERR_ARG;
    if (c->build_ip_weights()) return IBG_ERR_CUDA;
    const size_t n = kind < 2 ? c->S : c->F;
    cudaMemcpyAsync(c->d_ip_tmp, a, sizeof(double) * n, cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(c->d_ip_tmp + c->F, b, sizeof(double) * n, cudaMemcpyHostToDevice, c->st);
    return device_ip(c, kind, c->d_ip_tmp, c->d_ip_tmp + c->F, 1.0, ip);
}

int ibg_energy(ibg_context* c, double* energy) {
    if (!c || !energy) return IBG_ERR_ARG;
    if (c->build_ip_weights()) return IBG_ERR_CUDA;
    c->to64();
    return device_ip(c, 2, c->b64.q, c->b64.q, 0.5, energy);
}

int ibg_set_linearized(ibg_context* c, int period, const double* omega0, const double* q0) {
    if (!c || period < 0 || (period > 0 && (!omega0 || !q0))) return IBG_ERR_ARG;
    if (c->fp32) return c->fail(IBG_ERR_UNSUPPORTED, "ibg_set_linearized: the linearized forms run in FP64 only");
    cudaStreamSynchronize(c->st);
    c->release_variant();
    c->drop_graph();
    if (period == 0) return IBG_OK;  // back to NonlinearIBSolver
    if (c->alloc(&c->d_base_w, (size_t)period * c->S, false) || c->alloc(&c->d_base_q, (size_t)period * c->F, false))
        return IBG_ERR_CUDA;
    cudaMemcpy(c->d_base_w, omega0, sizeof(double) * period * c->S, cudaMemcpyHostToDevice);
    cudaMemcpy(c->d_base_q, q0, sizeof(double) * period * c->F, cudaMemcpyHostToDevice);
    c->nmode = 1;
    c->period = period;
    return c->cuda_check("ibg_set_linearized");
}

int ibg_set_adjoint(ibg_context* c, const double* omega0, const double* q0) {
    if (!c || !omega0 || !q0) return IBG_ERR_ARG;
    int s = ibg_set_linearized(c, 1, omega0, q0);
    if (s) return s;
    c->nmode = 3;
    return IBG_OK;
}

int ibg_set_sfd(ibg_context* c, double chi, double Delta, const double* omega_hat) {
    if (!c || !(Delta != 0.0)) return IBG_ERR_ARG;
    if (c->fp32) return c->fail(IBG_ERR_UNSUPPORTED, "ibg_set_sfd: selective frequency damping runs in FP64 only");
    cudaStreamSynchronize(c->st);
    c->release_variant();
    c->drop_graph();
    if (c->alloc(&c->d_what, c->S) || c->alloc(&c->d_rprev, c->S)) return IBG_ERR_CUDA;
    if (omega_hat) cudaMemcpy(c->d_what, omega_hat, sizeof(double) * c->S, cudaMemcpyHostToDevice);
    c->nmode = 2;
    c->sfd_chi = chi;
    c->sfd_Delta = Delta;
    c->sfd_rhs_saved = false;
    return c->cuda_check("ibg_set_sfd");
}

int ibg_get_sfd_state(ibg_context* c, double* omega_hat) {
    if (!c || !omega_hat) return IBG_ERR_ARG;
    if (c->nmode != 2) return c->fail(IBG_ERR_STATE, "ibg_get_sfd_state: selective frequency damping is not on");
    cudaMemcpyAsync(omega_hat, c->d_what, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_get_sfd_state");
    return IBG_OK;
}

int ibg_set_state(ibg_context* c, const double* omega, const double* q, const double* f, int timestep, double time) {
    if (!c) return IBG_ERR_ARG;
    Bulk<double>& B = c->b64;
    if (omega) cudaMemcpyAsync(B.w, omega, sizeof(double) * c->S, cudaMemcpyHostToDevice, c->st);
    else cudaMemsetAsync(B.w, 0, sizeof(double) * c->S, c->st);
    if (f) cudaMemcpyAsync(c->f, f, sizeof(double) * c->ncomp, cudaMemcpyHostToDevice, c->st);
    else cudaMemsetAsync(c->f, 0, sizeof(double) * c->ncomp, c->st);
    c->timestep = timestep;
    c->time = time;
    cudaMemcpyAsync(c->d_time, &c->time, sizeof(double), cudaMemcpyHostToDevice, c->st);
    cudaMemsetAsync(c->d_hist_count, 0, sizeof(int), c->st);
    cudaMemcpyAsync(c->d_ts0, &c->timestep, sizeof(int), cudaMemcpyHostToDevice, c->st);
    c->hist_steps = 0;
    if (q) {
        cudaMemcpyAsync(B.q, q, sizeof(double) * c->F, cudaMemcpyHostToDevice, c->st);
    } else {
        // model->updateOperators(x.time); model->refreshState(x) (src/ibpm.cc:300-305)
        if (c->ubf) c->frame_flow(0.0);
        if (c->moving) c->move_bodies(0.0);
        c->refresh<double>(B);
    }
    c->state_in_32 = false;
    c->to32();
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_set_state");
    return c->cuda_check("ibg_set_state");
}

int ibg_get_state(ibg_context* c, double* omega, double* q, double* f, int* timestep, double* time) {
    if (!c) return IBG_ERR_ARG;
    if (omega || q) c->to64();
    if (omega) cudaMemcpyAsync(omega, c->b64.w, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
    if (q) cudaMemcpyAsync(q, c->b64.q, sizeof(double) * c->F, cudaMemcpyDeviceToHost, c->st);
    if (f) cudaMemcpyAsync(f, c->f, sizeof(double) * c->ncomp, cudaMemcpyDeviceToHost, c->st);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_get_state");
    if (timestep) *timestep = c->timestep;
    if (time) *time = c->time;
    return c->cuda_check("ibg_get_state");
}

int ibg_get_boundary_force(ibg_context* c, double* f, int* timestep, double* time) {
    return ibg_get_state(c, nullptr, nullptr, f, timestep, time);
}

int ibg_update_operators(ibg_context* c, double time) {
    if (!c) return IBG_ERR_ARG;
    // the state's own time stays as it is
    const double keep = c->time;
    cudaMemcpyAsync(c->d_time, &time, sizeof(double), cudaMemcpyHostToDevice, c->st);
    if (c->ubf) c->frame_flow(0.0);
    if (c->moving) c->move_bodies(0.0);
    cudaMemcpyAsync(c->d_time, &keep, sizeof(double), cudaMemcpyHostToDevice, c->st);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_update_operators");
    return c->cuda_check("ibg_update_operators");
}

int ibg_set_moving_frame(ibg_context* c) {
    if (!c) return IBG_ERR_ARG;
    if (c->nbodies != 1)
        return c->fail(IBG_ERR_ARG, "ibg_set_moving_frame: the unsteady base flow needs exactly one body");
    if (c->ubf) return IBG_OK;
    BodyDev& b = c->h_bodies[0];
    if (b.motion == IBG_MOTION_NONE || b.motion == IBG_MOTION_FIXED) return IBG_OK;  // stationary: flag ignored
    if (c->chol_ready) return c->fail(IBG_ERR_STATE, "ibg_set_moving_frame: call before ibg_init");
    c->drop_graph();  // a captured step of the moving body no longer applies
    if (c->alloc(&c->d_bf, 1) || c->alloc(&c->d_bf_state, 1) || c->alloc(&c->d_bfv, 3) || c->alloc(&c->d_q0, c->F))
        return IBG_ERR_CUDA;
    // Geometry::transferMotion: the base flow takes a fresh copy of the motion, the body keeps none
    cudaMemcpyAsync(c->d_bf, &b, sizeof(BodyDev), cudaMemcpyHostToDevice, c->st);
    c->bf_xc = b.xc;
    c->bf_yc = b.yc;
    b.motion = IBG_MOTION_NONE;
    cudaMemcpyAsync(c->d_bodies, &b, sizeof(BodyDev), cudaMemcpyHostToDevice, c->st);
    c->moving = false;
    c->stateful = false;
    c->ubf = true;
    // the body at its reference points; BaseFlow's initial field is the uniform flow (src/BaseFlow.cc:65-78)
    c->move_bodies(0.0);
    const double uv[3] = {c->u0, c->v0, 0.0};
    cudaMemcpyAsync(c->d_bfv, uv, sizeof(uv), cudaMemcpyHostToDevice, c->st);
    launch_frame_flux(c->g, c->d_bfv, c->bf_xc, c->bf_yc, c->d_q0, c->st);
    launch_bcon_field(c->ncomp, c->slots, c->d_vel, c->d_q0, c->g.dx, c->d_b, c->st);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_set_moving_frame");
    return c->cuda_check("ibg_set_moving_frame");
}

int ibg_flux_to_velocity(ibg_context* c, double* u, double* v) {
    if (!c || !u || !v) return IBG_ERR_ARG;
    c->to64();
    // the FP64 node buffers of the nonlinear term are free between steps
    launch_flux_to_vel(c->g, c->b64.q, c->b64.U, c->b64.V, c->st);
    cudaMemcpyAsync(u, c->b64.U, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
    cudaMemcpyAsync(v, c->b64.V, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_flux_to_velocity");
    return c->cuda_check("ibg_flux_to_velocity");
}

int ibg_set_external_kinematics(ibg_context* c) {
    if (!c) return IBG_ERR_ARG;
    if (c->ubf) return c->fail(IBG_ERR_STATE, "ibg_set_external_kinematics: the moving frame carries the motion");
    if (!c->d_ext && c->alloc(&c->d_ext, (size_t)(kExtNow + 1) * 4 * c->npts)) return IBG_ERR_CUDA;
    // the current configuration becomes every slot until the caller writes them
    std::vector<double> h(4 * (size_t)c->npts);
    const int s = ibg_get_boundary(c, h.data(), h.data() + 2 * (size_t)c->npts);
    if (s) return s;
    for (int k = 0; k <= kExtNow; ++k)
        cudaMemcpyAsync(c->d_ext + (size_t)k * 4 * c->npts, h.data(), sizeof(double) * h.size(),
                        cudaMemcpyHostToDevice, c->st);
    c->ext_kin = true;
    c->moving = true;
    c->stateful = false;
    c->drop_graph();
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_set_external_kinematics");
    return c->cuda_check("ibg_set_external_kinematics");
}
int ibg_set_step_kinematics(ibg_context* c, int slot, const double* points, const double* velocities) {
    if (!c || !points || !velocities) return IBG_ERR_ARG;
    if (!c->ext_kin) return c->fail(IBG_ERR_STATE, "ibg_set_step_kinematics: call ibg_set_external_kinematics first");
    if (slot < -1 || slot >= c->sch.nsub) return c->fail(IBG_ERR_ARG, "ibg_set_step_kinematics: slot out of range");
    const size_t n2 = 2 * (size_t)c->npts;
    double* dst = c->d_ext + (size_t)(slot < 0 ? kExtNow : slot) * 2 * n2;
    cudaMemcpyAsync(dst, points, sizeof(double) * n2, cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(dst + n2, velocities, sizeof(double) * n2, cudaMemcpyHostToDevice, c->st);
    if (slot < 0) c->move_bodies(0.0, -1);
    return c->cuda_check("ibg_set_step_kinematics");
}
int ibg_get_boundary(ibg_context* c, double* points, double* velocities) {
    if (!c) return IBG_ERR_ARG;
    const size_t n = (size_t)c->npts;
    std::vector<double> h(4 * n);
    cudaMemcpyAsync(h.data(), c->d_pts, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, c->st);
    cudaMemcpyAsync(h.data() + 2 * n, c->d_vel, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, c->st);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_get_boundary");
    for (size_t p = 0; p < n; ++p)
        for (int d = 0; d < 2; ++d) {
            if (points) points[d * n + p] = h[2 * p + d];
            if (velocities) velocities[d * n + p] = h[2 * n + 2 * p + d];
        }
    return c->cuda_check("ibg_get_boundary");
}

int ibg_refresh_state(ibg_context* c) {
    if (!c) return IBG_ERR_ARG;
    if (c->fp32) {
        if (!c->state_in_32) c->to32();
        c->refresh<float>(c->b32);
    } else {
        c->refresh<double>(c->b64);
    }
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_refresh_state");
    return c->cuda_check("ibg_refresh_state");
}

int ibg_advance(ibg_context* c, int nsteps) {
    if (!c || nsteps < 0) return IBG_ERR_ARG;
    if (!c->moving && !c->chol_ready) return c->fail(IBG_ERR_STATE, "ibg_advance: call ibg_init (or ibg_load) first");
    const long long l0 = c->launches;
    if (c->fp32 && !c->state_in_32) c->to32();
    for (int n = 0; n < nsteps; ++n) {
        if (c->moving && c->prm.cg_precond == IBG_PRECOND_CHOLESKY &&
            (!c->chol_ready || c->steps_since_pc >= c->prm.pc_refresh)) {
            // rebuild the preconditioner at the current body configuration
            int s = c->build_operator();
            if (s) return s;
            c->steps_since_pc = 0;
        }
        ++c->steps_since_pc;
        if (c->old_saved && (!c->moving || c->prm.cg_graph)) {
            int gs = c->ensure_graph();
            if (gs) return gs;
            if (cudaGraphLaunch(c->graph, c->st) != cudaSuccess) return c->cuda_check("ibg_advance: graph launch");
            c->launches += c->graph_launches;
        } else {
            int s = c->enqueue_step();
            if (s) return s;
        }
        c->timestep += 1;
        c->time += c->prm.dt;
        c->hist_steps += 1;
    }
    c->last_launches = c->launches - l0;
    return c->cuda_check("ibg_advance");
}

int ibg_get_net_force(ibg_context* c, double* xf, double* yf) {
    if (!c) return IBG_ERR_ARG;
    std::vector<double> f(c->ncomp);
    int s = ibg_get_state(c, nullptr, nullptr, f.data(), nullptr, nullptr);
    if (s) return s;
    double sx = 0, sy = 0;
    for (int i = 0; i < c->npts; ++i) {
        sx += f[i];
        sy += f[c->npts + i];
    }
    const double dx2 = c->g.dx * c->g.dx;
    if (xf) *xf = sx * dx2;
    if (yf) *yf = sy * dx2;
    return IBG_OK;
}

int ibg_get_force_history(ibg_context* c, int n, double* xy) {
    if (!c || n < 0 || (n > 0 && !xy)) return IBG_ERR_ARG;
    long long have = c->hist_steps < kHistCap ? c->hist_steps : kHistCap;
    if (n > have) n = (int)have;
    std::vector<double> h(2 * (size_t)kHistCap);
    cudaMemcpyAsync(h.data(), c->d_hist, sizeof(double) * 2 * kHistCap, cudaMemcpyDeviceToHost, c->st);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_get_force_history");
    for (int k = 0; k < n; ++k) {
        long long step = c->hist_steps - n + k;
        long long slot = step % kHistCap;
        xy[2 * k] = h[2 * slot];
        xy[2 * k + 1] = h[2 * slot + 1];
    }
    return n;
}

int ibg_sizes(const ibg_context* c, long long* ns, long long* nf, int* nb) {
    if (!c) return IBG_ERR_ARG;
    if (ns) *ns = (long long)c->S;
    if (nf) *nf = (long long)c->F;
    if (nb) *nb = c->ncomp;
    return IBG_OK;
}

static void cg_device_stats(const ibg_context* c, int out[8]) {
    for (int i = 0; i < 8; ++i) out[i] = 0;
    if (!c->cg_flags) return;
    cudaMemcpyAsync(out, c->cg_flags, 8 * sizeof(int), cudaMemcpyDeviceToHost, c->st);
    cudaStreamSynchronize(c->st);
}

int ibg_cg_totals(const ibg_context* c, long long* iterations, long long* solves) {
    if (!c) return IBG_ERR_ARG;
    int d[8];
    cg_device_stats(c, d);
    if (iterations) *iterations = c->cg_total + d[3];
    if (solves) *solves = c->cg_solves + d[4];
    return IBG_OK;
}

int ibg_cg_stats(const ibg_context* c, int* last, int* mx, int* capped) {
    if (!c) return IBG_ERR_ARG;
    int d[8];
    cg_device_stats(c, d);
    if (d[4] > 0) {
        if (last) *last = d[1];
        if (mx) *mx = std::max(c->cg_max, d[5]);
        if (capped) *capped = c->cg_capped + d[6];
        return IBG_OK;
    }
    if (last) *last = c->cg_last;
    if (mx) *mx = c->cg_max;
    if (capped) *capped = c->cg_capped;
    return IBG_OK;
}

void* ibg_stream(const ibg_context* c) { return c ? (void*)c->st : nullptr; }
long long ibg_last_launch_count(const ibg_context* c) { return c ? c->last_launches : 0; }

namespace {
// kernel nodes of a graph, child graphs included; -1 if it holds a conditional node (whose body runs a
// data-dependent number of times)
long long count_kernel_nodes(cudaGraph_t gr) {
    size_t n = 0;
    if (cudaGraphGetNodes(gr, nullptr, &n) != cudaSuccess) return -1;
    std::vector<cudaGraphNode_t> nodes(n);
    if (n && cudaGraphGetNodes(gr, nodes.data(), &n) != cudaSuccess) return -1;
    long long k = 0;
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) != cudaSuccess) return -1;
        if (t == cudaGraphNodeTypeKernel) {
            ++k;
        } else if (t == cudaGraphNodeTypeGraph) {
            cudaGraph_t child = nullptr;
            if (cudaGraphChildGraphNodeGetGraph(nd, &child) != cudaSuccess) return -1;
            const long long c = count_kernel_nodes(child);
            if (c < 0) return -1;
            k += c;
        } else if (t == cudaGraphNodeTypeConditional) {
            return -1;
        }
    }
    return k;
}
}  // namespace

long long ibg_graph_kernel_nodes(ibg_context* c) {
    if (!c) return IBG_ERR_ARG;
    if (!c->graph_def) return IBG_ERR_STATE;
    return count_kernel_nodes(c->graph_def);
}

long long ibg_graph_launch_claim(const ibg_context* c) { return c ? c->graph_launches : 0; }

int ibg_pass_form_log(double* out, int max_rows) {
    std::lock_guard<std::mutex> lock(g_pform_mu);
    int r = 0;
    for (const auto& kv : g_pform) {
        if (out && r < max_rows) {
            double* o = out + 6 * r;
            for (int j = 0; j < 3; ++j) o[j] = kv.first[j];
            for (int j = 0; j < 3; ++j) o[3 + j] = kv.second[j];
        }
        ++r;
    }
    return r;
}

int ibg_sweep_form_log(double* out, int max_rows) {
    std::lock_guard<std::mutex> lock(g_sweep_mu);
    int r = 0;
    for (const auto& kv : g_sweep) {
        if (out && r < max_rows) {
            double* o = out + 7 * r;
            for (int j = 0; j < 4; ++j) o[j] = kv.first[j];
            for (int j = 0; j < 3; ++j) o[4 + j] = kv.second[j];
        }
        ++r;
    }
    return r;
}

int ibg_set_pass_form(ibg_context* c, int half_length) {
    if (!c) return IBG_ERR_ARG;
    cudaStreamSynchronize(c->st);
    int e = c->b64.poisson.grid ? c->b64.poisson.set_half(half_length != 0) : 0;
    for (int k = 0; k < 4 && !e; ++k)
        if (c->b64.helm[k].grid) e = c->b64.helm[k].set_half(half_length != 0);
    c->drop_graph();
    return e ? IBG_ERR_CUDA : IBG_OK;
}

int ibg_set_sweep_form(ibg_context* c, int edge_maps) {
    if (!c) return IBG_ERR_ARG;
    cudaStreamSynchronize(c->st);
    auto set = [&](auto& plan) { plan.edge_maps = edge_maps != 0; };
    set(c->b64.poisson);
    set(c->b32.poisson);
    for (int k = 0; k < 4; ++k) {
        set(c->b64.helm[k]);
        set(c->b32.helm[k]);
    }
    c->drop_graph();
    return IBG_OK;
}

// ---------------------------------------------------------------------------
// operator entry points
// ---------------------------------------------------------------------------
static int finish(ibg_context* c, const char* where) {
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check(where);
    return c->cuda_check(where);
}

int ibg_poisson_solve(ibg_context* c, const double* f, double* u) {
    if (!c || !f || !u) return IBG_ERR_ARG;
    Bulk<double>& B = c->b64;
    cudaMemcpyAsync(B.a, f, sizeof(double) * c->S, cudaMemcpyHostToDevice, c->st);
    B.poisson.solve(c->call<double>(B, B.a, B.psi, 1.0), c->st);
    cudaMemcpyAsync(u, B.psi, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
    return finish(c, "ibg_poisson_solve");
}

int ibg_helmholtz_solve(ibg_context* c, double alpha, const double* f, double* u) {
    if (!c || !f || !u) return IBG_ERR_ARG;
    EllipticPlan<double> h;
    if (h.init(&c->g, &c->fft, true, alpha, c->cosT)) return c->fail(IBG_ERR_CUDA, "helmholtz plan");
    Bulk<double>& B = c->b64;
    // the context's choices of the DST form and the sweep
    if (h.set_half(B.poisson.half)) return c->fail(IBG_ERR_CUDA, "helmholtz plan");
    h.edge_maps = B.poisson.edge_maps;
    cudaMemcpyAsync(B.a, f, sizeof(double) * c->S, cudaMemcpyHostToDevice, c->st);
    h.solve(c->call<double>(B, B.a, B.psi, 1.0), c->st);
    cudaMemcpyAsync(u, B.psi, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
    return finish(c, "ibg_helmholtz_solve");
}

int ibg_nonlinear(ibg_context* c, const double* q, const double* omega, double* out) {
    if (!c || !q || !omega || !out) return IBG_ERR_ARG;
    Bulk<double>& B = c->b64;
    cudaMemcpyAsync(B.qtmp, q, sizeof(double) * c->F, cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(B.a, omega, sizeof(double) * c->S, cudaMemcpyHostToDevice, c->st);
    launch_nonlinear<double>(c->g, B.qtmp, B.a, B.U, B.V, B.C, B.cc, 1, c->S, c->F, c->st);
    cudaMemcpyAsync(out, B.cc, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
    return finish(c, "ibg_nonlinear");
}

int ibg_laplacian(ibg_context* c, const double* fin, double* out) {
    if (!c || !fin || !out) return IBG_ERR_ARG;
    Bulk<double>& B = c->b64;
    cudaMemcpyAsync(B.a, fin, sizeof(double) * c->S, cudaMemcpyHostToDevice, c->st);
    launch_laplacian<double>(c->g, B.a, B.psi, c->st);
    cudaMemcpyAsync(out, B.psi, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
    return finish(c, "ibg_laplacian");
}

int ibg_model_B(ibg_context* c, const double* fb, double* omega) {
    if (!c || !fb || !omega) return IBG_ERR_ARG;
    cudaMemcpyAsync(c->btmp, fb, sizeof(double) * c->ncomp, cudaMemcpyHostToDevice, c->st);
    launch_smear_bf<double>(c->g, c->ncomp, c->slots, c->btmp, c->flux0, c->b64.Bf, 1.0, c->st);
    cudaMemcpyAsync(omega, c->b64.Bf, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
    return finish(c, "ibg_model_B");
}

int ibg_model_C(ibg_context* c, const double* omega, double* fb) {
    if (!c || !omega || !fb) return IBG_ERR_ARG;
    Bulk<double>& B = c->b64;
    cudaMemcpyAsync(B.a, omega, sizeof(double) * c->S, cudaMemcpyHostToDevice, c->st);
    B.poisson.solve(c->call<double>(B, B.a, B.psi, -1.0), c->st);
    launch_reg_interp<double>(c->g, c->ncomp, c->slots, B.psi, c->S, 1, nullptr, c->btmp, 0, c->st);
    cudaMemcpyAsync(fb, c->btmp, sizeof(double) * c->ncomp, cudaMemcpyDeviceToHost, c->st);
    return finish(c, "ibg_model_C");
}

int ibg_reg_to_flux(ibg_context* c, const double* fb, double* q) {
    if (!c || !fb || !q) return IBG_ERR_ARG;
    const GridDev& g = c->g;
    cudaMemcpyAsync(c->btmp, fb, sizeof(double) * c->ncomp, cudaMemcpyHostToDevice, c->st);
    // level 0: sum of weight * f over the associations, times dx; every coarser level is zero
    launch_reg_smear(c->ncomp, c->slots, g.dx, c->btmp, c->flux0, c->st);
    launch_k(k_scale, (unsigned)((g.F1 + 255) / 256), 256, 0, c->st, (size_t)g.F1, (const double*)c->flux0, g.dx,
             c->b64.qtmp);
    launch_reg_zero(c->ncomp, c->slots, c->flux0, c->st);
    if (g.L > 1) cudaMemsetAsync(c->b64.qtmp + g.F1, 0, sizeof(double) * (c->F - g.F1), c->st);
    cudaMemcpyAsync(q, c->b64.qtmp, sizeof(double) * c->F, cudaMemcpyDeviceToHost, c->st);
    return finish(c, "ibg_reg_to_flux");
}
int ibg_reg_to_boundary(ibg_context* c, const double* qin, double* fb) {
    if (!c || !qin || !fb) return IBG_ERR_ARG;
    cudaMemcpyAsync(c->b64.qtmp, qin, sizeof(double) * c->g.F1, cudaMemcpyHostToDevice, c->st);
    launch_reg_gather(c->g, c->ncomp, c->slots, c->b64.qtmp, c->btmp, c->st);
    cudaMemcpyAsync(fb, c->btmp, sizeof(double) * c->ncomp, cudaMemcpyDeviceToHost, c->st);
    return finish(c, "ibg_reg_to_boundary");
}

int ibg_projection_solve(ibg_context* c, int k, const double* ain, const double* bin, double* omega, double* fio) {
    if (!c || !ain || !bin || !omega || !fio || k < 0 || k >= c->sch.nsub) return IBG_ERR_ARG;
    if (!c->moving && !c->chol_ready) return c->fail(IBG_ERR_STATE, "ibg_projection_solve: call ibg_init first");
    Bulk<double>& B = c->b64;
    cudaMemcpyAsync(B.a, ain, sizeof(double) * c->S, cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(c->btmp, bin, sizeof(double) * c->ncomp, cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(c->f, fio, sizeof(double) * c->ncomp, cudaMemcpyHostToDevice, c->st);
    int s = c->projection<double>(B, k, B.a, c->btmp);
    if (s) return s;
    c->state_in_32 = false;
    cudaMemcpyAsync(omega, B.w, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
    cudaMemcpyAsync(fio, c->f, sizeof(double) * c->ncomp, cudaMemcpyDeviceToHost, c->st);
    return finish(c, "ibg_projection_solve");
}

// ---------------------------------------------------------------------------
// standalone multi-domain elliptic solvers (PoissonSolver / HelmholtzSolver)
// ---------------------------------------------------------------------------
struct ibg_elliptic {
    GridDev g{};
    size_t S = 0;
    FftTables fft;
    CosTables cosT;
    EllipticPlan<double> plan;
    double *f = nullptr, *u = nullptr, *rc = nullptr, *tbuf = nullptr, *sweep = nullptr;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    std::string err;
    ~ibg_elliptic() {
        double* p[] = {f, u, rc, tbuf, sweep};
        for (double* x : p)
            if (x) cudaFree(x);
        fft.release();
        cosT.release();
        if (own_stream && st) cudaStreamDestroy(st);
    }
};
namespace {
thread_local std::string g_elliptic_error;
}

int ibg_elliptic_create(const ibg_grid* grid, int helmholtz, double alpha, void* cuda_stream, ibg_elliptic** out) {
    if (!grid || !out) {
        g_elliptic_error = "ibg_elliptic_create: null argument";
        return IBG_ERR_ARG;
    }
    *out = nullptr;
    const ibg_grid& G = *grid;
    if (G.nx < 4 || G.ny < 4 || G.ngrid < 1 || G.ngrid > 16 || !(G.length > 0) ||
        (G.ngrid > 1 && (G.nx % 2 || G.ny % 2))) {
        g_elliptic_error = "ibg_elliptic_create: invalid grid";
        return IBG_ERR_ARG;
    }
    if (!fft_supported(2 * G.nx) || !fft_supported(2 * G.ny)) {
        g_elliptic_error = "ibg_elliptic_create: 2*nx and 2*ny must factor into primes <= 13";
        return IBG_ERR_UNSUPPORTED;
    }
    auto* e = new ibg_elliptic();
    GridDev& g = e->g;
    g.nx = G.nx;
    g.ny = G.ny;
    g.L = G.ngrid;
    g.nxe = (int)floor(G.nx / 4 + 0.5);  // src/Grid.h:60-62 with zero shift
    g.nye = (int)floor(G.ny / 4 + 0.5);
    g.NI = G.nx - 1;
    g.NJ = G.ny - 1;
    g.N1 = g.NI * g.NJ;
    g.nXf = (G.nx + 1) * G.ny;
    g.F1 = 2 * G.nx * G.ny + G.nx + G.ny;
    g.dx = G.length / G.nx;
    g.x0 = G.xoffset;
    g.y0 = G.yoffset;
    e->S = (size_t)g.L * g.N1;
    if (cuda_stream) {
        e->st = (cudaStream_t)cuda_stream;
    } else if (cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete e;
        g_elliptic_error = "ibg_elliptic_create: no CUDA device or stream creation failed";
        return IBG_ERR_CUDA;
    } else {
        e->own_stream = true;
    }
    int s = e->fft.init(2 * g.ny, 2 * g.nx);
    if (!s) s = e->cosT.init(g.nx, g.ny, g.nxe, g.nye);
    if (!s && g.L > 1) s = e->cosT.build_edge_maps(g.nx, g.ny, g.nxe, g.nye, e->fft);
    if (!s) s = e->plan.init(&e->g, &e->fft, helmholtz != 0, alpha, e->cosT);
    const size_t sw = sweep_doubles(g.nx, g.ny, g.L);
    if (!s && (cudaMalloc(&e->f, sizeof(double) * e->S) || cudaMalloc(&e->u, sizeof(double) * e->S) ||
               cudaMalloc(&e->rc, sizeof(double) * e->S) || cudaMalloc(&e->tbuf, sizeof(double) * e->S) ||
               cudaMalloc(&e->sweep, sizeof(double) * sw)))
        s = IBG_ERR_CUDA;
    if (s) {
        g_elliptic_error = "ibg_elliptic_create: set-up or device allocation failed";
        delete e;
        return s;
    }
    *out = e;
    return IBG_OK;
}
int ibg_elliptic_solve(ibg_elliptic* e, const double* f, double* u) {
    if (!e || !f || !u) return IBG_ERR_ARG;
    cudaMemcpyAsync(e->f, f, sizeof(double) * e->S, cudaMemcpyHostToDevice, e->st);
    SolveCall<double> c{};
    c.f = e->f;
    c.u = e->u;
    c.rc = e->rc;
    c.tbuf = e->tbuf;
    c.sweep = e->sweep;
    c.bstride = e->S;
    c.batch = 1;
    c.in_scale = 1.0;
    int s = e->plan.solve(c, e->st);
    cudaMemcpyAsync(u, e->u, sizeof(double) * e->S, cudaMemcpyDeviceToHost, e->st);
    const cudaError_t ce = cudaStreamSynchronize(e->st);
    if (s || ce != cudaSuccess) {
        e->err = std::string("ibg_elliptic_solve: ") + cudaGetErrorString(ce != cudaSuccess ? ce : cudaGetLastError());
        return IBG_ERR_CUDA;
    }
    return IBG_OK;
}
int ibg_elliptic_destroy(ibg_elliptic* e) {
    if (!e) return IBG_ERR_ARG;
    if (e->st) cudaStreamSynchronize(e->st);
    delete e;
    return IBG_OK;
}
const char* ibg_elliptic_last_error(const ibg_elliptic* e) { return e ? e->err.c_str() : g_elliptic_error.c_str(); }

// ---------------------------------------------------------------------------
// ensembles: one graph whose independent branches are the members' steps
// ---------------------------------------------------------------------------
}  // extern "C"

struct ibg_ensemble {
    std::vector<ibg_context*> members;
    std::vector<cudaEvent_t> ev;  // one per member: orders member streams and the ensemble stream
    cudaEvent_t done = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t st = nullptr;
    long long launches_per_step = 0;
    // the host-state step (ibg_ensemble_advance_host): per member, copies in -> step -> copies out,
    // for the host arrays it was built with
    cudaGraph_t hgraph = nullptr;
    cudaGraphExec_t hexec = nullptr;
    std::vector<const void*> hptrs;
    std::vector<cudaGraph_t> hparts;  // the members' captured copy-in and copy-out graphs
    long long hlaunches_per_step = 0;
    std::string err;
    void drop_host_graph() {
        if (hexec) cudaGraphExecDestroy(hexec);
        if (hgraph) cudaGraphDestroy(hgraph);
        for (cudaGraph_t g : hparts) cudaGraphDestroy(g);
        hexec = nullptr;
        hgraph = nullptr;
        hparts.clear();
        hptrs.clear();
        hlaunches_per_step = 0;
    }
    ~ibg_ensemble() {
        drop_host_graph();
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (cudaEvent_t x : ev) cudaEventDestroy(x);
        if (done) cudaEventDestroy(done);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {
thread_local std::string g_ens_error;
}

extern "C" {

int ibg_ensemble_create(int n, ibg_context* const* members, ibg_ensemble** out) {
    if (n < 1 || !members || !out) {
        g_ens_error = "ibg_ensemble_create: no members";
        return IBG_ERR_ARG;
    }
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        ibg_context* c = members[i];
        if (!c) {
            g_ens_error = "ibg_ensemble_create: null member";
            return IBG_ERR_ARG;
        }
        if (c->moving || c->ubf) {
            g_ens_error = "ibg_ensemble_create: members must have fixed bodies and a steady base flow";
            return IBG_ERR_UNSUPPORTED;
        }
        if (!c->chol_ready) {
            g_ens_error = "ibg_ensemble_create: call ibg_init (or ibg_load) on every member first";
            return IBG_ERR_STATE;
        }
    }
    auto* e = new ibg_ensemble();
    e->members.assign(members, members + n);
    for (ibg_context* c : e->members) c->use_rule_shapes();
    e->ev.assign(n, nullptr);
    bool ok = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaGraphCreate(&e->graph, 0) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < n && ok; ++i) ok = cudaEventCreateWithFlags(&e->ev[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        g_ens_error = "ibg_ensemble_create: stream or graph creation failed";
        delete e;
        return IBG_ERR_CUDA;
    }
    *out = e;
    return IBG_OK;
}

static int ensemble_build(ibg_ensemble* e) {
    for (ibg_context* c : e->members) {
        int s = c->ensure_graph();
        if (s) {
            e->err = std::string("member capture: ") + c->err;
            return s;
        }
        cudaStreamSynchronize(c->st);
        cudaGraphNode_t node;
        if (cudaGraphAddChildGraphNode(&node, e->graph, nullptr, 0, c->graph_def) != cudaSuccess) {
            e->err = "ibg_ensemble: adding a member graph failed";
            return IBG_ERR_CUDA;
        }
        e->launches_per_step += c->graph_launches;
    }
    if (cudaGraphInstantiate(&e->exec, e->graph, 0) != cudaSuccess) {
        e->err = "ibg_ensemble: graph instantiation failed";
        return IBG_ERR_CUDA;
    }
    return IBG_OK;
}

int ibg_ensemble_advance(ibg_ensemble* e, int nsteps) {
    if (!e || nsteps < 0) return IBG_ERR_ARG;
    if (!e->exec) {
        // a member's first step runs on its own (start-up of the N_prev history);
        // if any member has not stepped yet, every member takes that first step alone
        bool fresh = false;
        for (ibg_context* c : e->members) fresh = fresh || !c->old_saved;
        if (fresh && nsteps > 0) {
            for (ibg_context* c : e->members) {
                int s = ibg_advance(c, 1);
                if (s) {
                    e->err = std::string("member first step: ") + c->err;
                    return s;
                }
            }
            --nsteps;
        }
        if (fresh && nsteps == 0) return IBG_OK;
        int s = ensemble_build(e);
        if (s) return s;
    }
    // the ensemble step follows whatever the members' own streams have queued ...
    for (size_t i = 0; i < e->members.size(); ++i) {
        cudaEventRecord(e->ev[i], e->members[i]->st);
        cudaStreamWaitEvent(e->st, e->ev[i], 0);
    }
    for (int n = 0; n < nsteps; ++n) {
        if (cudaGraphLaunch(e->exec, e->st) != cudaSuccess) {
            e->err = std::string("ibg_ensemble_advance: ") + cudaGetErrorString(cudaGetLastError());
            return IBG_ERR_CUDA;
        }
        for (ibg_context* c : e->members) {
            c->timestep += 1;
            c->time += c->prm.dt;
            c->hist_steps += 1;
            c->last_launches = c->graph_launches;
        }
    }
    // ... and whatever the members do next follows the ensemble step
    cudaEventRecord(e->done, e->st);
    for (ibg_context* c : e->members) cudaStreamWaitEvent(c->st, e->done, 0);
    return IBG_OK;
}

// the host-state step graph: member i's branch copies omega[i], q[i], f[i] in (and converts them to
// FP32 for an FP32 member), runs the member's captured step and copies the state back out
static int ensemble_build_host(ibg_ensemble* e, double* const* omega, double* const* q, double* const* f) {
    e->drop_host_graph();
    if (cudaGraphCreate(&e->hgraph, 0) != cudaSuccess) {
        e->err = "ibg_ensemble_advance_host: graph creation failed";
        return IBG_ERR_CUDA;
    }
    for (size_t i = 0; i < e->members.size(); ++i) {
        ibg_context* c = e->members[i];
        cudaGraph_t pre = nullptr, post = nullptr;
        const long long l0 = c->launches;
        if (cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return c->cuda_check("capture");
        cudaMemcpyAsync(c->b64.w, omega[i], sizeof(double) * c->S, cudaMemcpyHostToDevice, c->st);
        cudaMemcpyAsync(c->b64.q, q[i], sizeof(double) * c->F, cudaMemcpyHostToDevice, c->st);
        cudaMemcpyAsync(c->f, f[i], sizeof(double) * c->ncomp, cudaMemcpyHostToDevice, c->st);
        c->to32();
        if (cudaStreamEndCapture(c->st, &pre) != cudaSuccess) return c->cuda_check("capture end");
        e->hparts.push_back(pre);
        if (cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return c->cuda_check("capture");
        c->to64();
        cudaMemcpyAsync(omega[i], c->b64.w, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
        cudaMemcpyAsync(q[i], c->b64.q, sizeof(double) * c->F, cudaMemcpyDeviceToHost, c->st);
        cudaMemcpyAsync(f[i], c->f, sizeof(double) * c->ncomp, cudaMemcpyDeviceToHost, c->st);
        if (cudaStreamEndCapture(c->st, &post) != cudaSuccess) return c->cuda_check("capture end");
        e->hparts.push_back(post);
        const long long conv = c->fp32 ? 4 : 0;  // k_convert in and out, two arrays each
        c->launches = l0;
        cudaGraphNode_t n0, n1, n2;
        if (cudaGraphAddChildGraphNode(&n0, e->hgraph, nullptr, 0, pre) != cudaSuccess ||
            cudaGraphAddChildGraphNode(&n1, e->hgraph, &n0, 1, c->graph_def) != cudaSuccess ||
            cudaGraphAddChildGraphNode(&n2, e->hgraph, &n1, 1, post) != cudaSuccess) {
            e->err = "ibg_ensemble_advance_host: adding a member's nodes failed";
            return IBG_ERR_CUDA;
        }
        e->hlaunches_per_step += c->graph_launches + conv;
        e->hptrs.push_back(omega[i]);
        e->hptrs.push_back(q[i]);
        e->hptrs.push_back(f[i]);
    }
    if (cudaGraphInstantiate(&e->hexec, e->hgraph, 0) != cudaSuccess) {
        e->err = "ibg_ensemble_advance_host: graph instantiation failed";
        return IBG_ERR_CUDA;
    }
    return IBG_OK;
}

int ibg_ensemble_advance_host(ibg_ensemble* e, int nsteps, double* const* omega, double* const* q,
                              double* const* f) {
    if (!e || nsteps < 0 || !omega || !q || !f) return IBG_ERR_ARG;
    const size_t n = e->members.size();
    for (size_t i = 0; i < n; ++i) {
        if (!omega[i] || !q[i] || !f[i]) return IBG_ERR_ARG;
        // the copies are captured into a graph: the host arrays must be page-locked
        const void* p3[3] = {omega[i], q[i], f[i]};
        for (const void* p : p3) {
            cudaPointerAttributes at{};
            if (cudaPointerGetAttributes(&at, p) != cudaSuccess || at.type != cudaMemoryTypeHost) {
                cudaGetLastError();
                e->err = "ibg_ensemble_advance_host: the State arrays must be page-locked host memory "
                         "(cudaHostAlloc / cudaHostRegister)";
                return IBG_ERR_ARG;
            }
        }
    }
    for (ibg_context* c : e->members)
        if (!c->old_saved) {
            e->err = "ibg_ensemble_advance_host: advance the ensemble by ibg_ensemble_advance first";
            return IBG_ERR_STATE;
        }
    if (!e->exec) {
        int s = ensemble_build(e);
        if (s) return s;
    }
    bool same = e->hexec && e->hptrs.size() == 3 * n;
    for (size_t i = 0; same && i < n; ++i)
        same = e->hptrs[3 * i] == omega[i] && e->hptrs[3 * i + 1] == q[i] && e->hptrs[3 * i + 2] == f[i];
    if (!same) {
        cudaStreamSynchronize(e->st);
        for (ibg_context* c : e->members) cudaStreamSynchronize(c->st);
        int s = ensemble_build_host(e, omega, q, f);
        if (s) {
            e->drop_host_graph();
            return s;
        }
    }
    for (size_t i = 0; i < n; ++i) {
        cudaEventRecord(e->ev[i], e->members[i]->st);
        cudaStreamWaitEvent(e->st, e->ev[i], 0);
    }
    for (int k = 0; k < nsteps; ++k) {
        if (cudaGraphLaunch(e->hexec, e->st) != cudaSuccess) {
            e->err = std::string("ibg_ensemble_advance_host: ") + cudaGetErrorString(cudaGetLastError());
            return IBG_ERR_CUDA;
        }
        for (ibg_context* c : e->members) {
            c->timestep += 1;
            c->time += c->prm.dt;
            c->hist_steps += 1;
            c->last_launches = c->graph_launches + (c->fp32 ? 4 : 0);
        }
    }
    if (cudaStreamSynchronize(e->st) != cudaSuccess) {
        e->err = std::string("ibg_ensemble_advance_host: ") + cudaGetErrorString(cudaGetLastError());
        return IBG_ERR_CUDA;
    }
    for (ibg_context* c : e->members) c->state_in_32 = c->fp32;
    return IBG_OK;
}

long long ibg_ensemble_host_launches_per_step(const ibg_ensemble* e) { return e ? e->hlaunches_per_step : 0; }

// drop the parent graph (rebuilt from the members' captures at the next advance)
static int ensemble_reset(ibg_ensemble* e) {
    e->drop_host_graph();
    if (e->exec) cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
    if (e->graph) cudaGraphDestroy(e->graph);
    e->graph = nullptr;
    e->launches_per_step = 0;
    if (cudaGraphCreate(&e->graph, 0) != cudaSuccess) {
        e->err = "ibg_ensemble: graph creation failed";
        return IBG_ERR_CUDA;
    }
    return IBG_OK;
}

namespace {
struct EnsTune {
    int nx, ny, levels, pairs, threads;
    double ms;  // ensemble step time with this class's chosen shape
};
}  // namespace

int ibg_ensemble_autotune(ibg_ensemble* e, int steps_per_trial, int* out, int max_rows) {
    if (!e || steps_per_trial < 1) return IBG_ERR_ARG;
    for (ibg_context* c : e->members)
        if (!c->old_saved) {
            e->err = "ibg_ensemble_autotune: advance the ensemble by ibg_ensemble_advance first";
            return IBG_ERR_STATE;
        }
    // size classes (grid shape), largest first; every member starts from two pairs and 128 threads
    std::map<std::pair<int, int>, std::vector<ibg_context*>> cls;
    for (ibg_context* c : e->members) cls[{c->g.nx, c->g.ny}].push_back(c);
    std::vector<std::pair<int, int>> order;
    for (auto& kv : cls) order.push_back(kv.first);
    std::sort(order.begin(), order.end(), [](auto a, auto b) { return a.first * a.second > b.first * b.second; });
    // (four pairs per CTA, 4/128 and 4/256, lost to 2/128 on the whole 64-member set: not tried here)
    const int cand[][2] = {{2, 128}, {1, 128}, {2, 256}, {1, 256}, {2, 96}};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto trial = [&](double& ms) -> int {
        int s = ensemble_reset(e);
        if (s) return s;
        s = ibg_ensemble_advance(e, 1);  // captures and instantiates; not timed
        if (s) return s;
        cudaEventRecord(e0, e->st);
        s = ibg_ensemble_advance(e, steps_per_trial);
        if (s) return s;
        cudaEventRecord(e1, e->st);
        if (cudaEventSynchronize(e1) != cudaSuccess) return IBG_ERR_CUDA;
        float v = 0.f;
        cudaEventElapsedTime(&v, e0, e1);
        ms = v / steps_per_trial;
        return IBG_OK;
    };
    auto set_class = [&](const std::vector<ibg_context*>& ms, int P, int T) -> int {
        cudaStreamSynchronize(e->st);
        int r = IBG_OK;
        for (ibg_context* c : ms) {
            cudaStreamSynchronize(c->st);
            const int q = c->set_shapes(P, T, false);
            if (q && !r) r = q;
        }
        return r;
    };
    std::vector<EnsTune> log;
    double best_all = 0.0;
    int s = trial(best_all);
    for (size_t ci = 0; ci < order.size() && !s; ++ci) {
        const auto& ms = cls[order[ci]];
        int bp = 2, bt = 128;
        double best = best_all;
        for (const auto& cd : cand) {
            if (cd[0] == 2 && cd[1] == 128) continue;
            if (set_class(ms, cd[0], cd[1])) continue;  // a shape too large for this grid class
            double t = 0.0;
            s = trial(t);
            if (s) break;
            if (t < 0.99 * best) {
                best = t;
                bp = cd[0];
                bt = cd[1];
            }
        }
        if (s) break;
        s = set_class(ms, bp, bt);
        if (s) break;
        best_all = best;
        log.push_back({order[ci].first, order[ci].second, ms[0]->g.L, bp, bt, best});
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!s) s = ensemble_reset(e);
    if (s) return s;
    if (out)
        for (size_t r = 0; r < log.size() && (int)r < max_rows; ++r) {
            int* o = out + 5 * r;
            o[0] = log[r].nx;
            o[1] = log[r].ny;
            o[2] = (int)std::lround(1000.0 * log[r].ms);  // us per ensemble step after this class
            o[3] = log[r].pairs;
            o[4] = log[r].threads;
        }
    return (int)log.size();
}

int ibg_ensemble_set_shapes(ibg_ensemble* e, int pairs_per_cta, int threads, int edge_maps) {
    if (!e || pairs_per_cta < 0 || pairs_per_cta > 4 || pairs_per_cta == 3 ||
        (pairs_per_cta > 0 && (threads < 32 || threads > 512 || threads % 32)))
        return IBG_ERR_ARG;
    cudaStreamSynchronize(e->st);
    int st = IBG_OK;
    for (ibg_context* c : e->members) {
        cudaStreamSynchronize(c->st);
        const int q = c->set_shapes(pairs_per_cta, threads, edge_maps != 0);
        if (q && !st) st = q;
    }
    // the parent graph is rebuilt from the members' new captures at the next advance
    e->drop_host_graph();
    if (e->exec) cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
    if (e->graph) cudaGraphDestroy(e->graph);
    e->graph = nullptr;
    e->launches_per_step = 0;
    if (cudaGraphCreate(&e->graph, 0) != cudaSuccess) {
        e->err = "ibg_ensemble_set_shapes: graph creation failed";
        return IBG_ERR_CUDA;
    }
    if (st) e->err = "ibg_ensemble_set_shapes: the shape needs more shared memory than a CTA may take for some "
                     "member; those members keep their previous shape";
    return st;
}

int ibg_ensemble_destroy(ibg_ensemble* e) {
    if (!e) return IBG_ERR_ARG;
    cudaStreamSynchronize(e->st);
    delete e;
    return IBG_OK;
}

long long ibg_ensemble_kernel_nodes(const ibg_ensemble* e) {
    if (!e) return IBG_ERR_ARG;
    if (!e->exec) return IBG_ERR_STATE;
    return count_kernel_nodes(e->graph);
}
void* ibg_ensemble_stream(const ibg_ensemble* e) { return e ? (void*)e->st : nullptr; }
long long ibg_ensemble_launches_per_step(const ibg_ensemble* e) { return e ? e->launches_per_step : 0; }
const char* ibg_ensemble_last_error(const ibg_ensemble* e) { return e ? e->err.c_str() : g_ens_error.c_str(); }

// ---------------------------------------------------------------------------
// learned preconditioner: data from the solver, training, parameters
// ---------------------------------------------------------------------------
namespace ibg {
__global__ void k_gather_rows(int nrows, long width, const int* __restrict__ idx, const float* __restrict__ src,
                              float* __restrict__ dst) {
    pdl_enter();
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nrows * width) return;
    const long r = t / width, c = t % width;
    dst[t] = src[(size_t)idx[r] * width + c];
}
}  // namespace ibg

static int lpc_ensure(ibg_context* c) {
    if (c->lpc.params) return IBG_OK;
    if (c->lpc.init(c->npts, c->h_nbr, c->h_cnt)) return c->fail(IBG_ERR_CUDA, "learned preconditioner set-up failed");
    if (c->prm.cg_precond == IBG_PRECOND_LEARNED)
        for (int k = 0; k < c->sch.nsub; ++k)
            if (!c->Mi[k] && c->alloc(&c->Mi[k], (size_t)c->ncomp * c->ncomp)) return IBG_ERR_CUDA;
    return IBG_OK;
}

size_t ibg_lpc_num_params(void) { return lpc_num_params(); }

int ibg_lpc_generate(ibg_context* c, int nconfig, double t0, double t1, float* geom, float* mb) {
    if (!c || nconfig < 1 || !geom || !mb) return IBG_ERR_ARG;
    if (lpc_ensure(c)) return IBG_ERR_CUDA;
    const int P = c->npts, m = c->ncomp, k = c->sch.nsub - 1;
    std::vector<double> Mh((size_t)m * m);
    const double keep_time = c->time;
    int status = IBG_OK;
    // the sampled configurations are not part of the body's motion history
    cudaMemcpyAsync(c->d_mstate_keep, c->d_mstate, sizeof(MotionState) * c->nbodies, cudaMemcpyDeviceToDevice, c->st);
    for (int cf = 0; cf < nconfig && !status; ++cf) {
        const double t = nconfig == 1 ? t0 : t0 + (t1 - t0) * cf / (nconfig - 1);
        cudaMemcpyAsync(c->d_time, &t, sizeof(double), cudaMemcpyHostToDevice, c->st);
        c->move_bodies(0.0);
        status = c->build_m(k);
        if (status) break;
        c->lpc.geometry(c->d_pts, c->lb, c->st);
        cudaMemcpyAsync(geom + (size_t)cf * 4 * P, c->lpc.geom, sizeof(float) * 4 * P, cudaMemcpyDeviceToHost, c->st);
        cudaMemcpyAsync(Mh.data(), c->bs_M, sizeof(double) * Mh.size(), cudaMemcpyDeviceToHost, c->st);
        if (cudaStreamSynchronize(c->st) != cudaSuccess) {
            status = c->cuda_check("ibg_lpc_generate");
            break;
        }
        // bs_M holds column j of M at j m: M[i][j] = Mh[j m + i]
        float* out = mb + (size_t)cf * m * m;
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) out[(size_t)i * m + j] = (float)(Mh[(size_t)j * m + i] / c->beta[k]);
    }
    // back to the current configuration
    cudaMemcpyAsync(c->d_mstate, c->d_mstate_keep, sizeof(MotionState) * c->nbodies, cudaMemcpyDeviceToDevice, c->st);
    cudaMemcpyAsync(c->d_time, &keep_time, sizeof(double), cudaMemcpyHostToDevice, c->st);
    c->move_bodies(0.0);
    if (cudaStreamSynchronize(c->st) != cudaSuccess && !status) status = c->cuda_check("ibg_lpc_generate");
    return status;
}

// device copies of a training set
struct LpcData {
    float* g = nullptr;
    float* mb = nullptr;
    void release() {
        if (g) cudaFree(g);
        if (mb) cudaFree(mb);
        g = mb = nullptr;
    }
};

static int lpc_upload(ibg_context* c, int n, const float* geom, const float* mb, LpcData& d) {
    const size_t P = c->npts, m = c->ncomp;
    if (c->alloc(&d.g, n * 4 * P, false) || c->alloc(&d.mb, n * m * m, false)) return IBG_ERR_CUDA;
    cudaMemcpy(d.g, geom, sizeof(float) * n * 4 * P, cudaMemcpyHostToDevice);
    cudaMemcpy(d.mb, mb, sizeof(float) * n * m * m, cudaMemcpyHostToDevice);
    return IBG_OK;
}

int ibg_lpc_loss_grad(ibg_context* c, int nconfig, const float* geom, const float* mb, const float* params,
                      float* loss, float* grad) {
    if (!c || nconfig < 1 || !geom || !mb) return IBG_ERR_ARG;
    if (lpc_ensure(c)) return IBG_ERR_CUDA;
    const size_t np = lpc_num_params();
    LpcData d;
    float* dgrad = nullptr;
    if (lpc_upload(c, nconfig, geom, mb, d) || (grad && c->alloc(&dgrad, np))) {
        d.release();
        return IBG_ERR_CUDA;
    }
    if (params) {
        cudaMemcpy(c->lpc.params, params, sizeof(float) * np, cudaMemcpyHostToDevice);
        c->lpc.refresh_bf16(c->st);
    }
    float l = 0.f;
    int s = c->lpc.loss_grad(nconfig, d.g, d.mb, &l, dgrad, c->tws, c->st);
    if (!s && grad) cudaMemcpy(grad, dgrad, sizeof(float) * np, cudaMemcpyDeviceToHost);
    if (loss) *loss = l;
    d.release();
    if (dgrad) cudaFree(dgrad);
    if (s) return c->fail(s, "ibg_lpc_loss_grad: training work arrays");
    return c->cuda_check("ibg_lpc_loss_grad");
}

int ibg_lpc_train(ibg_context* c, int nconfig, const float* geom, const float* mb, int epochs, int batch, float lr,
                  unsigned int seed, float* loss_hist) {
    if (!c || nconfig < 1 || epochs < 1 || batch < 1 || !geom || !mb || !(lr > 0.f)) return IBG_ERR_ARG;
    if (lpc_ensure(c)) return IBG_ERR_CUDA;
    const int P = c->npts, m = c->ncomp;
    const size_t np = lpc_num_params();
    if (batch > nconfig) batch = nconfig;
    // operator scale c0: mean diagonal of M / beta over the data (stored after the weights)
    double dsum = 0.0;
    for (int cf = 0; cf < nconfig; ++cf)
        for (int i = 0; i < m; ++i) dsum += mb[(size_t)cf * m * m + (size_t)i * m + i];
    const float c0 = (float)(dsum / ((double)nconfig * m));
    if (!(c0 > 0.f)) return c->fail(IBG_ERR_ARG, "ibg_lpc_train: the operators' diagonal is not positive");
    cudaMemcpy(c->lpc.params + (np - 1), &c0, sizeof(float), cudaMemcpyHostToDevice);
    LpcData d;
    float *bg = nullptr, *bm = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
    int* didx = nullptr;
    auto cleanup = [&]() {
        d.release();
        float* f[] = {bg, bm, grad, m1, m2};
        for (float* x : f)
            if (x) cudaFree(x);
        if (didx) cudaFree(didx);
    };
    if (lpc_upload(c, nconfig, geom, mb, d) || c->alloc(&bg, (size_t)batch * 4 * P) ||
        c->alloc(&bm, (size_t)batch * m * m) || c->alloc(&grad, np) || c->alloc(&m1, np) || c->alloc(&m2, np) ||
        c->alloc(&didx, batch)) {
        cleanup();
        return IBG_ERR_CUDA;
    }
    std::mt19937 rng(seed);
    std::vector<int> perm(nconfig);
    for (int i = 0; i < nconfig; ++i) perm[i] = i;
    int step = 0, s = IBG_OK;
    const int total = epochs * (nconfig / batch);
    for (int ep = 0; ep < epochs && !s; ++ep) {
        std::shuffle(perm.begin(), perm.end(), rng);
        double acc = 0;
        int nb = 0;
        for (int b0 = 0; b0 + batch <= nconfig && !s; b0 += batch) {
            cudaMemcpyAsync(didx, perm.data() + b0, sizeof(int) * batch, cudaMemcpyHostToDevice, c->st);
            const long wg = 4L * P, wm = (long)m * m;
            launch_k(k_gather_rows, (unsigned)((batch * wg + 255) / 256), 256, 0, c->st, batch, wg, didx, d.g, bg);
            launch_k(k_gather_rows, (unsigned)((batch * wm + 255) / 256), 256, 0, c->st, batch, wm, didx, d.mb, bm);
            float l = 0.f;
            s = c->lpc.loss_grad(batch, bg, bm, &l, grad, c->tws, c->st);
            if (s) break;
            // cosine learning-rate decay to lr / 20; c0 stays fixed
            const float lr_t = lr * (0.05f + 0.95f * 0.5f * (1.f + std::cos(3.14159265f * step / std::max(1, total))));
            adam_step((long)np - 1, c->lpc.params, grad, m1, m2, lr_t, ++step, c->st);
            acc += l;
            ++nb;
        }
        if (loss_hist) loss_hist[ep] = (float)(acc / std::max(1, nb));
    }
    c->lpc.refresh_bf16(c->st);
    if (cudaStreamSynchronize(c->st) != cudaSuccess && !s) s = c->cuda_check("ibg_lpc_train");
    cleanup();
    if (s) return c->fail(s, "ibg_lpc_train failed");
    c->lpc_ready = true;
    c->drop_graph();  // a step captured before ran with the identity preconditioner
    return c->cuda_check("ibg_lpc_train");
}

int ibg_lpc_get_params(ibg_context* c, float* p, size_t n) {
    if (!c || !p || n != lpc_num_params()) return IBG_ERR_ARG;
    if (lpc_ensure(c)) return IBG_ERR_CUDA;
    cudaMemcpy(p, c->lpc.params, sizeof(float) * n, cudaMemcpyDeviceToHost);
    return c->cuda_check("ibg_lpc_get_params");
}

int ibg_lpc_set_params(ibg_context* c, const float* p, size_t n) {
    if (!c || !p || n != lpc_num_params()) return IBG_ERR_ARG;
    if (lpc_ensure(c)) return IBG_ERR_CUDA;
    cudaMemcpy(c->lpc.params, p, sizeof(float) * n, cudaMemcpyHostToDevice);
    c->lpc.refresh_bf16(c->st);
    cudaStreamSynchronize(c->st);
    c->lpc_ready = true;
    c->drop_graph();
    return c->cuda_check("ibg_lpc_set_params");
}

int ibg_lpc_apply(ibg_context* c, int k, const double* r, double* z, float* geom) {
    if (!c || !r || !z || k < 0 || k >= c->sch.nsub) return IBG_ERR_ARG;
    if (lpc_ensure(c)) return IBG_ERR_CUDA;
    const int m = c->ncomp;
    double *dr = nullptr, *dz = nullptr;
    double* K[4] = {nullptr, nullptr, nullptr, nullptr};
    int s = c->alloc(&dr, m) || c->alloc(&dz, m);
    for (int q = 0; q < c->sch.nsub && !s; ++q) s = c->alloc(&K[q], (size_t)m * m);
    if (!s) {
        cudaMemcpyAsync(dr, r, sizeof(double) * m, cudaMemcpyHostToDevice, c->st);
        c->lpc.geometry(c->d_pts, c->lb, c->st);
        c->lpc.operators(c->sch.nsub, c->beta, K, c->st);
        minv_apply(m, K[k], dr, dz, c->st);
        cudaMemcpyAsync(z, dz, sizeof(double) * m, cudaMemcpyDeviceToHost, c->st);
        if (geom) cudaMemcpyAsync(geom, c->lpc.geom, sizeof(float) * 4 * c->npts, cudaMemcpyDeviceToHost, c->st);
        cudaStreamSynchronize(c->st);
    }
    if (dr) cudaFree(dr);
    if (dz) cudaFree(dz);
    for (double* x : K)
        if (x) cudaFree(x);
    if (s) return IBG_ERR_CUDA;
    return c->cuda_check("ibg_lpc_apply");
}

int ibg_set_dst_gemm(ibg_context* c, int on) {
    if (!c) return IBG_ERR_ARG;
    if (!c->b32.ready) return c->fail(IBG_ERR_STATE, "ibg_set_dst_gemm: the context has no FP32 plans");
    c->set_dst_gemm(on != 0);
    return IBG_OK;
}
int ibg_dst_gemm_status(ibg_context* c) {
    if (!c) return IBG_ERR_ARG;
    if (!c->sines.err) return 0;
    int e = 0;
    cudaMemcpyAsync(&e, c->sines.err, sizeof(int), cudaMemcpyDeviceToHost, c->st);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_dst_gemm_status");
    return e;
}
int ibg_solve_fp32(ibg_context* c, int substep, const double* f, double* u) {
    if (!c || !f || !u || substep < -1 || substep >= c->sch.nsub) return IBG_ERR_ARG;
    if (!c->b32.ready) return c->fail(IBG_ERR_STATE, "ibg_solve_fp32: the context has no FP32 plans");
    Bulk<float>& B = c->b32;
    Bulk<double>& D = c->b64;
    cudaMemcpyAsync(D.a, f, sizeof(double) * c->S, cudaMemcpyHostToDevice, c->st);
    launch_k(k_convert<double, float>, (unsigned)((c->S + 255) / 256), 256, 0, c->st, c->S, (const double*)D.a, B.a);
    const EllipticPlan<float>& p = substep < 0 ? B.poisson : B.helm[substep];
    p.solve(c->call<float>(B, B.a, B.psi, 1.0f), c->st);
    launch_k(k_convert<float, double>, (unsigned)((c->S + 255) / 256), 256, 0, c->st, c->S, (const float*)B.psi, D.psi);
    cudaMemcpyAsync(u, D.psi, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->st);
    return finish(c, "ibg_solve_fp32");
}
int ibg_lpc_set_tensor_cores(ibg_context* c, int on) {
    if (!c) return IBG_ERR_ARG;
    if (lpc_ensure(c)) return IBG_ERR_CUDA;
    c->lpc.tensor_cores = on != 0;
    c->drop_graph();
    return IBG_OK;
}
int ibg_lpc_status(ibg_context* c) {
    if (!c) return IBG_ERR_ARG;
    if (!c->lpc.err) return 0;
    int e = 0;
    cudaMemcpyAsync(&e, c->lpc.err, sizeof(int), cudaMemcpyDeviceToHost, c->st);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->cuda_check("ibg_lpc_status");
    return e;
}
int ibg_substep_beta(ibg_context* c, int k, double* beta) {
    if (!c || !beta || k < 0 || k >= c->sch.nsub) return IBG_ERR_ARG;
    *beta = c->beta[k];
    return IBG_OK;
}

int ibg_dst_form_log(double* out, int max_rows) {
    std::lock_guard<std::mutex> lock(g_form_mu);
    int k = 0;
    for (const auto& kv : g_form) {
        if (out && k < max_rows) {
            const double row[6] = {(double)kv.first[0], (double)kv.first[1], (double)kv.first[2], kv.second[0],
                                   kv.second[1], kv.second[2]};
            for (int q = 0; q < 6; ++q) out[6 * k + q] = row[q];
        }
        ++k;
    }
    return k;
}
int ibg_autotune_log(int* out, int max_rows) {
    const std::vector<TuneResult> r = tune_log();
    if (out)
        for (int k = 0; k < (int)r.size() && k < max_rows; ++k) {
            const TuneResult& t = r[k];
            const int row[8] = {t.wbytes, t.pass, t.m, t.nlines, t.nlev, t.P, t.threads, t.tw_smem};
            for (int q = 0; q < 8; ++q) out[8 * k + q] = row[q];
        }
    return (int)r.size();
}

long long ibg_run_kernel(ibg_context* c, int which, int reps) {
    if (!c || reps < 0 || which < 0 || which > 2) return IBG_ERR_ARG;
    const GridDev& g = c->g;
    // the transforms in the arithmetic the context's time step uses
    const bool f32 = c->fp32 || c->refined;
    for (int r = 0; r < reps; ++r) {
        if (which == 2) {
            Bulk<double>& B = c->b64;
            launch_nonlinear<double>(g, B.q, B.w, B.U, B.V, B.C, B.Nbuf[0], 1, c->S, c->F, c->st);
        } else if (f32) {
            Bulk<float>& B = c->b32;
            B.poisson.run_pass(which, which == 0 ? B.w : B.tbuf, B.tbuf, c->st);
        } else {
            Bulk<double>& B = c->b64;
            B.poisson.run_pass(which, which == 0 ? B.w : B.tbuf, B.tbuf, c->st);
        }
    }
    long long bytes;
    if (which == 0 || which == 1) bytes = (f32 ? 8LL : 16LL) * (long long)c->S;  // every level read + written once
    else bytes = 8LL * (long long)(c->F + c->S + 2 * c->S + c->F + c->F + c->S);   // q,w in; U,V; C; N
    if (c->cuda_check("ibg_run_kernel")) return IBG_ERR_CUDA;
    return bytes;
}

}  // extern "C"
