/*
 * fftw3.h -- project-written stand-in for the three FFTW 3 entry points that
 * the IBPM reference library calls (src/EllipticSolver2d.cc:34-35 plans a 2-D
 * RODFT00 x RODFT00 transform, :65 executes it, :39 destroys the plan).
 *
 * TEST INFRASTRUCTURE ONLY: this header and dst1_shim.c exist so that the
 * reference C++ sources can be compiled into the CPU oracle (oracle/_ref).
 * FFTW itself is not installed in this image.  Only the RODFT00 (DST-I)
 * kind is implemented; any other kind makes the planner return NULL.
 *
 * Semantics follow FFTW's published definition of RODFT00 (unnormalised):
 *   Y_k = 2 * sum_{j=0}^{n-1} X_j sin(pi (j+1)(k+1) / (n+1))   per dimension.
 */
#ifndef IBG_FFTW_SHIM_H
#define IBG_FFTW_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
    FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
    FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10
} fftw_r2r_kind;

#define FFTW_MEASURE    (0U)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PATIENT    (1U << 5)
#define FFTW_ESTIMATE   (1U << 6)

typedef struct ibg_shim_plan *fftw_plan;

fftw_plan fftw_plan_r2r_2d(int n0, int n1, double *in, double *out,
                           fftw_r2r_kind kind0, fftw_r2r_kind kind1,
                           unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif
#endif
