/*
 * dst1_shim.c -- FP64 DST-I (RODFT00) behind the FFTW 3 plan/execute API.
 *
 * TEST INFRASTRUCTURE ONLY (see fftw3.h).  Used to link the reference's
 * EllipticSolver2d (src/EllipticSolver2d.cc:26-85) into the CPU oracle.
 *
 * Algorithm: a DST-I of length N is read off the DFT of the odd extension
 * of length M = 2(N+1) (z_0 = z_{N+1} = 0, z_{M-k} = -z_k), whose DFT is
 * purely imaginary.  Two real lines a, b are packed as z = a + i b, so one
 * complex FFT yields both:  DST(a)_k = -Im Z_{k+1},  DST(b)_k = Re Z_{k+1}.
 * The complex FFT is an iterative Stockham autosort FFT with mixed radices
 * (4, 2, 3, 5 and a generic prime-length DFT for any other factor), with
 * twiddles w_M^k = exp(-2 pi i k / M) tabulated once per plan with libm.
 */
#include "fftw3.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int m;              /* complex FFT length = 2 (n + 1) */
    int nfac;
    int fac[64];
    double *twr, *twi;  /* w_m^k, k < m */
} cfft_t;

struct ibg_shim_plan {
    int n0, n1;
    double *in, *out;
    cfft_t f0, f1;
    double *zr, *zi, *wr, *wi;   /* work, length max(m0, m1) */
};

static void cfft_init(cfft_t *p, int m) {
    int n = m, r;
    const int pref[4] = {4, 2, 3, 5};
    p->m = m;
    p->nfac = 0;
    for (int t = 0; t < 4; ++t) {
        r = pref[t];
        while (n % r == 0) { p->fac[p->nfac++] = r; n /= r; }
    }
    for (r = 7; n > 1; r += 2)
        while (n % r == 0) { p->fac[p->nfac++] = r; n /= r; }
    p->twr = (double *)malloc(sizeof(double) * m);
    p->twi = (double *)malloc(sizeof(double) * m);
    const double pi = 3.14159265358979323846264338327950288;
    for (int k = 0; k < m; ++k) {
        double a = -2.0 * pi * (double)k / (double)m;
        p->twr[k] = cos(a);
        p->twi[k] = sin(a);
    }
}

static void cfft_free(cfft_t *p) { free(p->twr); free(p->twi); }

/* Stockham autosort FFT; result ends in (xr, xi). */
static void cfft_exec(const cfft_t *p, double *xr, double *xi, double *wr, double *wi) {
    const int m = p->m;
    double *sr = xr, *si = xi, *dr = wr, *di = wi;
    int ns = 1;
    double vr[64], vi[64], orr[64], oi[64];
    for (int s = 0; s < p->nfac; ++s) {
        const int R = p->fac[s];
        const int mr = m / R;
        const int tstep = m / (ns * R);
        const int rstep = m / R;
        for (int j = 0; j < mr; ++j) {
            const int jm = j % ns;
            for (int q = 0; q < R; ++q) {
                double ar = sr[j + q * mr], ai = si[j + q * mr];
                int ti = (jm * q * tstep) % m;
                double cr = p->twr[ti], ci = p->twi[ti];
                vr[q] = ar * cr - ai * ci;
                vi[q] = ar * ci + ai * cr;
            }
            if (R == 2) {
                orr[0] = vr[0] + vr[1]; oi[0] = vi[0] + vi[1];
                orr[1] = vr[0] - vr[1]; oi[1] = vi[0] - vi[1];
            } else if (R == 4) {
                double t0r = vr[0] + vr[2], t0i = vi[0] + vi[2];
                double t1r = vr[0] - vr[2], t1i = vi[0] - vi[2];
                double t2r = vr[1] + vr[3], t2i = vi[1] + vi[3];
                double t3r = vr[1] - vr[3], t3i = vi[1] - vi[3];
                orr[0] = t0r + t2r; oi[0] = t0i + t2i;
                orr[2] = t0r - t2r; oi[2] = t0i - t2i;
                /* -i * t3 */
                orr[1] = t1r + t3i; oi[1] = t1i - t3r;
                orr[3] = t1r - t3i; oi[3] = t1i + t3r;
            } else {
                for (int pp = 0; pp < R; ++pp) {
                    double accr = 0.0, acci = 0.0;
                    for (int q = 0; q < R; ++q) {
                        int ti = ((pp * q) % R) * rstep;
                        double cr = p->twr[ti], ci = p->twi[ti];
                        accr += vr[q] * cr - vi[q] * ci;
                        acci += vr[q] * ci + vi[q] * cr;
                    }
                    orr[pp] = accr; oi[pp] = acci;
                }
            }
            const int idxd = (j / ns) * ns * R + jm;
            for (int pp = 0; pp < R; ++pp) {
                dr[idxd + pp * ns] = orr[pp];
                di[idxd + pp * ns] = oi[pp];
            }
        }
        double *t;
        t = sr; sr = dr; dr = t;
        t = si; si = di; di = t;
        ns *= R;
    }
    if (sr != xr) {
        memcpy(xr, sr, sizeof(double) * m);
        memcpy(xi, si, sizeof(double) * m);
    }
}

/* DST-I of `count` lines of length n; element k of line l at base[l*ls + k*es]. */
static void dst_lines(struct ibg_shim_plan *P, const cfft_t *f, int n, int count,
                      const double *src, double *dst, int ls, int es) {
    const int m = f->m;
    for (int l = 0; l < count; l += 2) {
        const int two = (l + 1 < count);
        const double *a = src + (size_t)l * ls;
        const double *b = two ? src + (size_t)(l + 1) * ls : NULL;
        P->zr[0] = 0.0; P->zi[0] = 0.0;
        P->zr[n + 1] = 0.0; P->zi[n + 1] = 0.0;
        for (int k = 0; k < n; ++k) {
            double ar = a[(size_t)k * es];
            double bi = two ? b[(size_t)k * es] : 0.0;
            P->zr[k + 1] = ar;       P->zi[k + 1] = bi;
            P->zr[m - 1 - k] = -ar;  P->zi[m - 1 - k] = -bi;
        }
        cfft_exec(f, P->zr, P->zi, P->wr, P->wi);
        double *oa = dst + (size_t)l * ls;
        double *ob = two ? dst + (size_t)(l + 1) * ls : NULL;
        for (int k = 0; k < n; ++k) {
            oa[(size_t)k * es] = -P->zi[k + 1];
            if (two) ob[(size_t)k * es] = P->zr[k + 1];
        }
    }
}

fftw_plan fftw_plan_r2r_2d(int n0, int n1, double *in, double *out,
                           fftw_r2r_kind kind0, fftw_r2r_kind kind1,
                           unsigned flags) {
    (void)flags;
    if (kind0 != FFTW_RODFT00 || kind1 != FFTW_RODFT00 || n0 < 1 || n1 < 1)
        return NULL;
    struct ibg_shim_plan *P = (struct ibg_shim_plan *)calloc(1, sizeof(*P));
    P->n0 = n0; P->n1 = n1; P->in = in; P->out = out;
    cfft_init(&P->f0, 2 * (n0 + 1));
    cfft_init(&P->f1, 2 * (n1 + 1));
    int mm = P->f0.m > P->f1.m ? P->f0.m : P->f1.m;
    P->zr = (double *)malloc(sizeof(double) * mm);
    P->zi = (double *)malloc(sizeof(double) * mm);
    P->wr = (double *)malloc(sizeof(double) * mm);
    P->wi = (double *)malloc(sizeof(double) * mm);
    return P;
}

void fftw_execute(const fftw_plan p) {
    struct ibg_shim_plan *P = p;
    /* along dimension 1 (contiguous rows), then along dimension 0 (columns) */
    dst_lines(P, &P->f1, P->n1, P->n0, P->in, P->out, P->n1, 1);
    dst_lines(P, &P->f0, P->n0, P->n1, P->out, P->out, 1, P->n1);
}

void fftw_destroy_plan(fftw_plan p) {
    struct ibg_shim_plan *P = p;
    if (!P) return;
    cfft_free(&P->f0); cfft_free(&P->f1);
    free(P->zr); free(P->zi); free(P->wr); free(P->wi);
    free(P);
}
