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

#ifdef __cplusplus
}
#endif
#endif
