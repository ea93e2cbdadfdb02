// ibg_lpc.cuh -- the learned preconditioner network (lpc.cu).
#pragma once
#include <vector>

#include "ibg_internal.cuh"

namespace ibg {

size_t lpc_num_params();

// body layout for the geometry features
struct LpcBodies {
    int n = 0;
    const int* body_of = nullptr;  // per point
    int* start = nullptr;          // per body: first point
    int* len = nullptr;            // per body: number of points
    int* closed = nullptr;         // per body: 1 if the points form a closed curve
};

// FP32 training work arrays, grown on demand (rows = configurations x P^2 point pairs)
struct TrainScratch {
    long rows = 0;
    int cfgs = 0;
    float *gbar = nullptr, *X = nullptr, *H1 = nullptr, *H2 = nullptr, *KO = nullptr, *K = nullptr, *E = nullptr;
    float *dK = nullptr, *dKO = nullptr, *dH2 = nullptr, *dH1 = nullptr, *lossc = nullptr;
    float* part = nullptr;  // split-K partial products of the weight gradients
    void release();
};

struct Lpc {
    int P = 0;
    float* params = nullptr;   // FP32 master weights (+ the operator scale c0 as the last entry)
    void* wbf = nullptr;       // BF16 inference weights: W1 (256 x 19), W2 transposed (256 x 256), W3 (4 x 256)
    int *nbr = nullptr, *cnt = nullptr;
    float* geom = nullptr;     // current geometry features (P x 4)
    float* gbar = nullptr;     // their neighbour means (P x 4)
    float* kraw = nullptr;     // network output per point pair (P^2 x 4)
    void* w2op = nullptr;      // W2 in BF16 as the tensor-core kernel's B operand (lpc_tc.cu)
    int* err = nullptr;        // set by the tensor-core kernel when a bounded wait ran out
    bool tensor_cores = true;  // inference on tcgen05 (else the CUDA-core kernel)
    int num_sms = 148;
    int init(int npts, const std::vector<int>& nbr_h, const std::vector<int>& cnt_h);
    void release();
    void refresh_bf16(cudaStream_t st);
    // geometry features of the current body configuration
    void geometry(const double* pts, const LpcBodies& bodies, cudaStream_t st) const;
    // K_k = sym(net) / (c0 beta_k) for every sub-step k < nsub into Kout[k] (m x m, FP64), at the
    // geometry last computed by geometry()
    void operators(int nsub, const double* beta, double* const* Kout, cudaStream_t st) const;
    // mean loss |K Mn - I|_F^2 / m over B configurations (device arrays: g [B][P][4], Mb [B][m][m]
    // = M / beta); gradient (lpc_num_params floats, the c0 entry 0) when grad != nullptr
    int loss_grad(int B, const float* g, const float* Mb, float* loss, float* grad, TrainScratch& ws,
                  cudaStream_t st) const;
};

// tensor-core inference (lpc_tc.cu)
int lpc_infer_tc_setup();
void lpc_w2_operand(const float* params, void* w2op, cudaStream_t st);
void lpc_infer_tc(int P, const float* g, const float* gbar, const float* params, const void* w2op, float* kraw,
                  int* err, int num_sms, cudaStream_t st);

void adam_step(long n, float* p, const float* g, float* m1, float* m2, float lr, int t, cudaStream_t st);

}  // namespace ibg
