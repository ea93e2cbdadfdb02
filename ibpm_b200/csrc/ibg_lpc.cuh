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

struct TrainScratch {
    int rows = 0;
    float *A = nullptr, *s = nullptr, *h1 = nullptr, *C = nullptr, *h2 = nullptr, *out = nullptr, *dout = nullptr;
    float *dh2 = nullptr, *dC = nullptr, *dh1 = nullptr;
    void release();
};

struct Lpc {
    int P = 0;
    float* params = nullptr;   // FP32 master weights
    void* wbf = nullptr;       // BF16 copy for inference
    int *nbr = nullptr, *cnt = nullptr;
    void *h1 = nullptr, *h2 = nullptr;  // BF16 inference activations
    float* geom = nullptr;     // current geometry features (P x 4)
    float* scale = nullptr;
    int init(int npts, const std::vector<int>& nbr_h, const std::vector<int>& cnt_h);
    void release();
    void refresh_bf16(cudaStream_t st);
    // z = (s/beta) net(r) for the current boundary (device pointers)
    void apply(const double* pts, const LpcBodies& bodies, const double* r, double* z, double beta,
               cudaStream_t st) const;
    // loss per sample over B samples (device arrays); gradient (kNParams floats) when grad != nullptr
    int loss_grad(int B, const float* g, const float* r, const float* t, float* loss_per_sample, float* grad,
                  TrainScratch& ws, cudaStream_t st) const;
};

void adam_step(long n, float* p, const float* g, float* m1, float* m2, float lr, int t, cudaStream_t st);

}  // namespace ibg
