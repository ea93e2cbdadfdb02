/* fftw3.h -- the one FFTW type the reference's headers name (EllipticSolver2d.h
 * keeps an fftw_plan member).  Used only where FFTW 3 itself is not installed:
 * the drop-in build calls no FFTW function (its transforms run on the GPU). */
#ifndef IBG_DROPIN_FFTW3_COMPAT_H
#define IBG_DROPIN_FFTW3_COMPAT_H
typedef struct fftw_plan_s* fftw_plan;
#endif
