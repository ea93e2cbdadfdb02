// ibg_force.cuh -- force-solve launchers (Cholesky, CG) and small utilities.
#pragma once
#include "ibg_internal.cuh"

namespace ibg {
int chol_factor(int m, const double* Mcol, double* Lr, double* Lc, double* diag, int* d_status, cudaStream_t st);
int chol_solve_prepare(int m);
void chol_solve(int m, const double* Lr, const double* Lc, const double* diag, const double* b, double* x,
                cudaStream_t st);
void chol_inverse(int m, const double* Lr, const double* Lc, const double* diag, double* Minv, cudaStream_t st);
void minv_apply(int m, const double* Minv, const double* b, double* y, cudaStream_t st);
void cg_begin(int m, const double* b, const double* Mx, double* r, double* d, double* scal, int* flags,
              cudaStream_t st);
void cg_update(int m, double* x, double* r, double* d, const double* q, double* scal, int* flags, cudaStream_t st);
void pcg_begin(int m, const double* b, const double* Mx, double* r, double* scal, int* flags, cudaStream_t st);
void pcg_begin2(int m, const double* r, double* z, double* d, double* scal, int* flags, cudaStream_t st);
void pcg_step1(int m, double* x, double* r, const double* d, const double* q, const double* z, double* zold,
               double* scal, int* flags, cudaStream_t st);
void pcg_step2(int m, const double* r, double* z, const double* zold, double* d, double* scal, int* flags,
               cudaStream_t st);
void net_force(int npts, const double* f, double dx2, double* out, cudaStream_t st);
void add_time(double* t, double dt, cudaStream_t st);
}  // namespace ibg
