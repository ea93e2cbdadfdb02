/*
 * ibpm_b200_diag.h -- measurement hooks of libibpm_b200.so (no reference
 * counterpart).  Not needed to run a simulation: they launch single kernels of
 * the time step so that their duration can be timed alone against the
 * hardware's roofline.
 */
#ifndef IBPM_B200_DIAG_H
#define IBPM_B200_DIAG_H

#include "ibpm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Launch one kernel of the time step `reps` times on the context's stream
 * (0: DST-I row pass of every level of one solve, 1: its column pass, 2: the
 * node-velocity kernel of the nonlinear term) and return the algorithmic bytes
 * one launch moves (each operand read once, each result written once), or a
 * negative status. */
IBG_API long long ibg_run_kernel(ibg_context* ctx, int which, int reps);

/* The learned preconditioner's network evaluation: on = 1 (the default) runs
 * its 256 x 256 layer on the tensor cores (tcgen05), on = 0 on the CUDA cores
 * (the two agree to BF16 rounding); the step graph is recaptured.
 * ibg_lpc_status returns 1 if a tensor-core evaluation ran out of a bounded
 * wait (its output is then not valid), 0 otherwise. */
IBG_API int ibg_lpc_set_tensor_cores(ibg_context* ctx, int on);

/* The FP32 plans' DST passes (the FP32 and FP32-refined forms): on = 1 runs
 * them as sine-matrix GEMMs on the tensor cores (tcgen05 kind::tf32, 3xTF32),
 * on = 0 as shared-memory FFTs (the default unless IBG_DST_GEMM=1 is set in the
 * environment when the context is created); the step graph is recaptured.
 * ibg_dst_gemm_status returns 1 if a GEMM pass ran out of a bounded wait.
 * ibg_solve_fp32 solves with the FP32 plan (substep -1: Poisson, k: the
 * Helmholtz problem of sub-step k) between FP64 host arrays. */
IBG_API int ibg_set_dst_gemm(ibg_context* ctx, int on);
IBG_API int ibg_dst_gemm_status(ibg_context* ctx);
IBG_API int ibg_solve_fp32(ibg_context* ctx, int substep, const double* f, double* u);
IBG_API int ibg_lpc_status(ibg_context* ctx);

/* The kernel nodes of the context's captured step graph (child graphs
 * included), to check the launch count the library reports for a step
 * (ibg_graph_launch_claim: the launches counted while the graph was
 * captured).  -1 when the graph holds a conditional node (the CG loop of
 * moving bodies, whose body runs a data-dependent number of times);
 * IBG_ERR_STATE before the first graph-launched step. */
IBG_API long long ibg_graph_kernel_nodes(ibg_context* ctx);
IBG_API long long ibg_graph_launch_claim(const ibg_context* ctx);
/* The coarse-to-fine sweep of every plan of the context: edge_maps = 1 applies
 * the precomputed edge maps (two launches per level transition, the default
 * of a single context), 0 the per-step line FFTs (inside the sums launch, the
 * default of ensemble members); the step graph is recaptured.  Results agree
 * to rounding. */
IBG_API int ibg_set_sweep_form(ibg_context* ctx, int edge_maps);
/* The autotuner's choice of that form per grid shape and precision (timed on
 * whole Poisson solves the first time a shape is created in the process; the
 * edge maps are kept unless the line FFTs are at least 3 % faster): up to
 * max_rows rows of 7 doubles {nx, ny, levels, bytes per word, edge maps chosen,
 * edge-map us, line-FFT us}; returns the number of shapes timed. */
IBG_API int ibg_sweep_form_log(double* out, int max_rows);
/* The autotuner's choice of the FP64 DST passes' form per grid shape (half-length FFTs or the odd
 * extension, timed on whole Poisson solves when a shape is first created; the half length is kept
 * unless the odd extension is at least 3 % faster): up to max_rows rows of 6 doubles {nx, ny, levels,
 * half length chosen, half-length us, odd-extension us}; returns the number of shapes timed. */
IBG_API int ibg_pass_form_log(double* out, int max_rows);
/* The form of every FP64 plan's DST passes and sweep lines: half_length = 1 the half-length FFTs, 0
 * the odd extension; the step graph is recaptured.  Results agree to rounding. */
IBG_API int ibg_set_pass_form(ibg_context* ctx, int half_length);
/* The same for an ensemble's graph (against ibg_ensemble_launches_per_step). */
IBG_API long long ibg_ensemble_kernel_nodes(const ibg_ensemble* ens);

#ifdef __cplusplus
}
#endif
#endif
