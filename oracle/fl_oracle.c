/*
 * fl_oracle.c -- FP64 CPU restatement of the FiberLab GMMNLSE hot path.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker + timed CPU baseline).  The CUDA
 * product never links this file.
 *
 * Follows, function by function:
 *   forward RHS      src/simulation/simulate_disp_mmf.jl:25-60
 *   forward driver   src/simulation/simulate_disp_mmf.jl:183-207
 *   adjoint RHS      src/simulation/sensitivity_disp_mmf.jl:32-79, 93-215
 *   adjoint gate     src/simulation/sensitivity_disp_mmf.jl:103-112, 237-240
 *   adjoint driver   src/simulation/sensitivity_disp_mmf.jl:309-332
 *   lab spectrum     src/fiberlab/propagation.jl:34-36
 *   RK4 cross-check  src/fiberlab/scalar_crosscheck.jl:38-67
 *   band cost/seed   src/fiberlab/physics_helpers.jl:222-232
 *   phase gradient   src/fiberlab/physics_models.jl:1041-1042
 *
 * The integrator is the third-party Tsit5 (OrdinaryDiffEqTsit5 1.12.0 /
 * OrdinaryDiffEqCore 3.33.0, called at simulate_disp_mmf.jl:190 and
 * sensitivity_disp_mmf.jl:328), restated from its published method:
 * Tsitouras (2011) 7-stage FSAL 5(4) tableau and free 4th-order interpolant,
 * OrdinaryDiffEq's default PI step controller (beta1 = 7/(10*5),
 * beta2 = 2/(5*5), gamma = 9/10, qmin = 1/5, qmax = 10, qoldinit = 1e-4),
 * Hairer's initial-step heuristic, and the RMS error norm over
 * abstol + reltol*max(|u_n|, |u_{n+1}|).  The step sequence is not pinned by
 * any reference test.
 *
 * The FFT is an own iterative radix-2 transform with FFTW's conventions:
 * fft is unnormalised with exponent sign -1, ifft carries 1/N.
 */
#include "fl_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* ------------------------------------------------------------------------ */
/* FFT                                                                       */
/* ------------------------------------------------------------------------ */

typedef struct {
    int n;
    cplx *tw;   /* exp(-2 pi i k / n), k < n */
    cplx *work; /* n values of scratch (one plan per thread) */
} fft_plan;

static int plan_init(fft_plan *pl, int n) {
    pl->n = n;
    pl->tw = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    pl->work = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    if (!pl->tw || !pl->work) return -1;
    for (int k = 0; k < n; k++) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        pl->tw[k] = cos(a) + I * sin(a);
    }
    return 0;
}

static void plan_free(fft_plan *pl) {
    free(pl->tw);
    free(pl->work);
    pl->tw = NULL;
    pl->work = NULL;
}

static inline cplx cmul_(cplx a, cplx b) {
    return CMPLX(creal(a) * creal(b) - cimag(a) * cimag(b),
                 creal(a) * cimag(b) + cimag(a) * creal(b));
}

/* Radix-4 Stockham autosort pass (decimation in frequency) over
 * sub-sequences of length n at stride s, reading x and writing y, then the
 * rest of the transform on y; a final radix-2 pass when log2 n is odd.  eo
 * tracks which buffer must hold the result, so it ends in the caller's
 * array.  tw is the length-nfull table exp(-2 pi i k / nfull). */
static void stockham(int n, int s, int eo, cplx *x, cplx *y, const cplx *tw, int nfull) {
    if (n == 1) {
        if (eo)
            for (int q = 0; q < s; q++) y[q] = x[q];
        return;
    }
    if (n == 2) {
        cplx *z = eo ? y : x;
        for (int q = 0; q < s; q++) {
            const cplx a = x[q], b = x[q + s];
            z[q] = a + b;
            z[q + s] = a - b;
        }
        return;
    }
    const int n1 = n / 4, n2 = n / 2, n3 = n1 + n2, st = nfull / n;
    for (int p = 0; p < n1; p++) {
        const cplx w1 = tw[p * st], w2 = tw[2 * p * st], w3 = tw[3 * p * st];
        for (int q = 0; q < s; q++) {
            const cplx a = x[q + s * p], b = x[q + s * (p + n1)];
            const cplx c = x[q + s * (p + n2)], d = x[q + s * (p + n3)];
            const cplx apc = a + c, amc = a - c, bpd = b + d, bmd = b - d;
            const cplx jbmd = CMPLX(-cimag(bmd), creal(bmd)); /* i (b - d) */
            y[q + s * (4 * p + 0)] = apc + bpd;
            y[q + s * (4 * p + 1)] = cmul_(w1, amc - jbmd);
            y[q + s * (4 * p + 2)] = cmul_(w2, apc - bpd);
            y[q + s * (4 * p + 3)] = cmul_(w3, amc + jbmd);
        }
    }
    stockham(n1, 4 * s, !eo, y, x, tw, nfull);
}

/* unnormalised forward transform (exponent -1); the inverse is
 * conj(F(conj x)) / n (FFTW's conventions as used by the reference) */
static void fft_1d(const fft_plan *pl, cplx *a, int inverse) {
    const int n = pl->n;
    if (inverse)
        for (int i = 0; i < n; i++) a[i] = conj(a[i]);
    stockham(n, 1, 0, a, pl->work, pl->tw, n);
    if (inverse) {
        const double sc = 1.0 / (double)n;
        for (int i = 0; i < n; i++) a[i] = CMPLX(creal(a[i]) * sc, -cimag(a[i]) * sc);
    }
}

static void fft_cols(const fft_plan *pl, cplx *a, int ncols, int inverse) {
    for (int c = 0; c < ncols; c++) fft_1d(pl, a + (size_t)c * pl->n, inverse);
}

int orc_fft(orc_c64 *x, int nt, int ncols, int inverse) {
    if (nt < 2 || (nt & (nt - 1))) return ORC_EINVAL;
    fft_plan pl;
    if (plan_init(&pl, nt)) return ORC_ENOMEM;
    fft_cols(&pl, (cplx *)x, ncols, inverse);
    plan_free(&pl);
    return ORC_OK;
}

/* fftshift along dim 1 of an (nt, ncols) array: out[t] = in[(t + nt/2) % nt] */
static void fftshift_cols(const cplx *in, cplx *out, int nt, int ncols) {
    int h = nt / 2;
    for (int c = 0; c < ncols; c++) {
        const cplx *s = in + (size_t)c * nt;
        cplx *d = out + (size_t)c * nt;
        for (int t = 0; t < nt; t++) d[t] = s[(t + h) % nt];
    }
}

/* ------------------------------------------------------------------------ */
/* Workspaces                                                                */
/* ------------------------------------------------------------------------ */

typedef struct {
    const orc_problem *p;
    fft_plan pl;
    cplx *ep, *em;                /* nt*m */
    cplx *uw;                     /* nt*m */
    double *v, *w;                /* nt*m */
    double *dK;                   /* nt*m*m */
    cplx *dKc, *tmpMM;            /* nt*m*m */
    double *dR;                   /* nt*m*m */
    cplx *etaK, *etaR, *eta;      /* nt*m */
    /* adjoint extras */
    cplx *lw, *lt, *lwc, *ut, *utc, *uwi;   /* nt*m */
    double *d1;                   /* nt*m*m */
    cplx *d2, *gab, *gab2;        /* nt*m*m */
    double *dKR1;                 /* nt*m*m */
    cplx *sres, *gout, *t1, *t2, *t3, *t4; /* nt*m */
    cplx *ufwd;                   /* nt*m, interpolated forward field */
    cplx *sigma;                  /* nt */
} workspace;

#define G4(g, m, i, j, k, l) ((g)[(i) + (m) * ((j) + (m) * ((k) + (m) * (l)))])

static void ws_free(workspace *w) {
    plan_free(&w->pl);
    void *ptrs[] = {w->ep, w->em, w->uw, w->v, w->w, w->dK, w->dKc, w->tmpMM,
                    w->dR, w->etaK, w->etaR, w->eta, w->lw, w->lt, w->lwc,
                    w->ut, w->utc, w->uwi, w->d1, w->d2, w->gab, w->gab2,
                    w->dKR1, w->sres, w->gout, w->t1, w->t2, w->t3, w->t4,
                    w->ufwd, w->sigma};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
    memset(w, 0, sizeof(*w));
}

static int ws_init(workspace *w, const orc_problem *p, int adjoint) {
    memset(w, 0, sizeof(*w));
    w->p = p;
    size_t n1 = (size_t)p->nt * p->m, n2 = n1 * p->m;
    if (plan_init(&w->pl, p->nt)) return -1;
    int bad = 0;
#define ALLOC(f, T, n)                              \
    do {                                            \
        w->f = (T *)calloc((n), sizeof(T));         \
        if (!w->f) bad = 1;                         \
    } while (0)
    ALLOC(ep, cplx, n1); ALLOC(em, cplx, n1); ALLOC(uw, cplx, n1);
    ALLOC(v, double, n1); ALLOC(w, double, n1);
    ALLOC(dK, double, n2); ALLOC(dKc, cplx, n2); ALLOC(tmpMM, cplx, n2);
    ALLOC(dR, double, n2);
    ALLOC(etaK, cplx, n1); ALLOC(etaR, cplx, n1); ALLOC(eta, cplx, n1);
    if (adjoint) {
        ALLOC(lw, cplx, n1); ALLOC(lt, cplx, n1); ALLOC(lwc, cplx, n1);
        ALLOC(ut, cplx, n1); ALLOC(utc, cplx, n1); ALLOC(uwi, cplx, n1);
        ALLOC(d1, double, n2); ALLOC(d2, cplx, n2); ALLOC(gab, cplx, n2);
        ALLOC(gab2, cplx, n2); ALLOC(dKR1, double, n2);
        ALLOC(sres, cplx, n1); ALLOC(gout, cplx, n1);
        ALLOC(t1, cplx, n1); ALLOC(t2, cplx, n1); ALLOC(t3, cplx, n1);
        ALLOC(t4, cplx, n1); ALLOC(ufwd, cplx, n1);
        ALLOC(sigma, cplx, (size_t)p->nt);
        if (!bad) {
            /* exp.(1im * π * repeat([0, 1], Nt ÷ 2)) */
            for (int t = 0; t < p->nt; t++)
                w->sigma[t] = cexp(I * M_PI * (double)(t & 1));
        }
    }
#undef ALLOC
    if (bad) {
        ws_free(w);
        return -1;
    }
    return 0;
}

static void phase_factors(workspace *w, double z) {
    const orc_problem *p = w->p;
    size_t n1 = (size_t)p->nt * p->m;
    for (size_t i = 0; i < n1; i++) {
        double a = p->D[i] * z;
        w->ep[i] = cos(a) + I * sin(a);
        double b = -p->D[i] * z;
        w->em[i] = cos(b) + I * sin(b);
    }
}

/* Raman convolution of the (nt, m*m) real sequences src:
 * dst = real(fftshift(ifft(hR .* fft(src)), 1)) */
static void raman_conv(workspace *w, const double *src, double *dst) {
    const orc_problem *p = w->p;
    int nt = p->nt, mm = p->m * p->m;
    size_t n2 = (size_t)nt * mm;
    for (size_t i = 0; i < n2; i++) w->dKc[i] = src[i];
    fft_cols(&w->pl, w->dKc, mm, 0);
    const cplx *hR = (const cplx *)p->hR;
    for (int c = 0; c < mm; c++)
        for (int t = 0; t < nt; t++) w->dKc[(size_t)c * nt + t] *= hR[t];
    fft_cols(&w->pl, w->dKc, mm, 1);
    fftshift_cols(w->dKc, w->tmpMM, nt, mm);
    for (size_t i = 0; i < n2; i++) dst[i] = creal(w->tmpMM[i]);
}

/* ------------------------------------------------------------------------ */
/* Forward RHS: simulate_disp_mmf.jl:25-60                                  */
/* ------------------------------------------------------------------------ */

static void rhs_forward_ws(workspace *w, double z, const cplx *u, cplx *du) {
    const orc_problem *p = w->p;
    int nt = p->nt, m = p->m;
    size_t n1 = (size_t)nt * m;
    phase_factors(w, z);
    for (size_t i = 0; i < n1; i++) w->uw[i] = w->ep[i] * u[i];
    fft_cols(&w->pl, w->uw, m, 0);
    for (size_t i = 0; i < n1; i++) {
        w->v[i] = creal(w->uw[i]);
        w->w[i] = cimag(w->uw[i]);
    }
    /* δKt[t,i,j] = γ[i,j,k,l] * (v[t,k] v[t,l] + w[t,k] w[t,l]) */
    for (int j = 0; j < m; j++)
        for (int i = 0; i < m; i++) {
            double *dk = w->dK + (size_t)nt * (i + m * j);
            for (int t = 0; t < nt; t++) dk[t] = 0.0;
            for (int l = 0; l < m; l++)
                for (int k = 0; k < m; k++) {
                    double g = G4(p->gamma, m, i, j, k, l);
                    if (g == 0.0) continue;
                    const double *vk = w->v + (size_t)nt * k, *vl = w->v + (size_t)nt * l;
                    const double *wk = w->w + (size_t)nt * k, *wl = w->w + (size_t)nt * l;
                    for (int t = 0; t < nt; t++) dk[t] += g * (vk[t] * vl[t] + wk[t] * wl[t]);
                }
        }
    /* αK, βK, ηK */
    for (int i = 0; i < m; i++)
        for (int t = 0; t < nt; t++) {
            double a = 0.0, b = 0.0;
            for (int j = 0; j < m; j++) {
                double d = w->dK[(size_t)nt * (i + m * j) + t];
                a += d * w->v[(size_t)nt * j + t];
                b += d * w->w[(size_t)nt * j + t];
            }
            w->etaK[(size_t)nt * i + t] = (a + I * b) * p->one_m_fR;
        }
    /* Raman */
    raman_conv(w, w->dK, w->dR);
    for (int i = 0; i < m; i++)
        for (int t = 0; t < nt; t++) {
            double a = 0.0, b = 0.0;
            for (int j = 0; j < m; j++) {
                double d = w->dR[(size_t)nt * (i + m * j) + t];
                a += d * w->v[(size_t)nt * j + t];
                b += d * w->w[(size_t)nt * j + t];
            }
            w->etaR[(size_t)nt * i + t] = a + I * b;
        }
    for (size_t i = 0; i < n1; i++) w->eta[i] = w->etaK[i] + w->etaR[i];
    fft_cols(&w->pl, w->eta, m, 1);
    for (int i = 0; i < m; i++)
        for (int t = 0; t < nt; t++) w->eta[(size_t)nt * i + t] *= p->selfsteep[t];
    for (size_t i = 0; i < n1; i++) du[i] = I * w->em[i] * w->eta[i];
}

/* ------------------------------------------------------------------------ */
/* Adjoint RHS: sensitivity_disp_mmf.jl:32-79 and helpers :93-215           */
/* ------------------------------------------------------------------------ */

/* calc_γ_a_b!: out[t,i,j] = Σ_{l,k} (a[t,l] b[t,k]) γ[l,k,i,j] */
static void calc_gamma_a_b(const orc_problem *p, const cplx *a, const cplx *b, cplx *out) {
    int nt = p->nt, m = p->m;
    for (int j = 0; j < m; j++)
        for (int i = 0; i < m; i++) {
            cplx *o = out + (size_t)nt * (i + m * j);
            for (int t = 0; t < nt; t++) o[t] = 0.0;
            for (int k = 0; k < m; k++)
                for (int l = 0; l < m; l++) {
                    double g = G4(p->gamma, m, l, k, i, j);
                    if (g == 0.0) continue;
                    const cplx *al = a + (size_t)nt * l, *bk = b + (size_t)nt * k;
                    for (int t = 0; t < nt; t++) {
                        double are = creal(al[t]), aim = cimag(al[t]);
                        double bre = creal(bk[t]), bim = cimag(bk[t]);
                        double re = are * bre - aim * bim;
                        double im = are * bim + aim * bre;
                        o[t] += (re * g) + I * (im * g);
                    }
                }
        }
}

/* calc_δs!: δ1 (|u|² part) and δ2 (u² part) with γ[l,k,i,j] */
static void calc_deltas(const orc_problem *p, const cplx *u, double *d1, cplx *d2) {
    int nt = p->nt, m = p->m;
    for (int j = 0; j < m; j++)
        for (int i = 0; i < m; i++) {
            double *o1 = d1 + (size_t)nt * (i + m * j);
            cplx *o2 = d2 + (size_t)nt * (i + m * j);
            for (int t = 0; t < nt; t++) {
                o1[t] = 0.0;
                o2[t] = 0.0;
            }
            for (int k = 0; k < m; k++)
                for (int l = 0; l < m; l++) {
                    double g = G4(p->gamma, m, l, k, i, j);
                    if (g == 0.0) continue;
                    const cplx *uk = u + (size_t)nt * k, *ul = u + (size_t)nt * l;
                    for (int t = 0; t < nt; t++) {
                        double vk = creal(uk[t]), wk = cimag(uk[t]);
                        double vl = creal(ul[t]), wl = cimag(ul[t]);
                        double a2 = vk * vl + wk * wl;
                        double sr = vk * vl - wk * wl;
                        double si = 2.0 * vk * wl;
                        o1[t] += a2 * g;
                        o2[t] += (sr * g) + I * (si * g);
                    }
                }
        }
}

static void rhs_adjoint_ws(workspace *w, double z, const cplx *lam, const cplx *ufwd, cplx *dlam) {
    const orc_problem *p = w->p;
    int nt = p->nt, m = p->m, mm = m * m;
    size_t n1 = (size_t)nt * m, n2 = n1 * m;
    const cplx *hR = (const cplx *)p->hR;
    phase_factors(w, z);
    /* λω = exp_D_p λ̃ω ; λω .*= τω ; λt = fft(λω) ; λωc = ifft(conj(λω)) */
    for (int i = 0; i < m; i++)
        for (int t = 0; t < nt; t++) {
            size_t q = (size_t)nt * i + t;
            w->lw[q] = w->ep[q] * lam[q];
            w->lw[q] *= p->selfsteep[t];
        }
    memcpy(w->lt, w->lw, sizeof(cplx) * n1);
    fft_cols(&w->pl, w->lt, m, 0);
    for (size_t q = 0; q < n1; q++) w->lwc[q] = conj(w->lw[q]);
    fft_cols(&w->pl, w->lwc, m, 1);
    /* forward field at z */
    for (size_t q = 0; q < n1; q++) w->uw[q] = w->ep[q] * ufwd[q];
    memcpy(w->ut, w->uw, sizeof(cplx) * n1);
    fft_cols(&w->pl, w->ut, m, 0);
    for (size_t q = 0; q < n1; q++) w->utc[q] = conj(w->ut[q]);
    memcpy(w->uwi, w->uw, sizeof(cplx) * n1);
    fft_cols(&w->pl, w->uwi, m, 1);          /* ifft_plan_M! * uω */
    /* Kerr operators */
    calc_deltas(p, w->ut, w->d1, w->d2);
    /* Raman convolution of δ1 */
    raman_conv(w, w->d1, w->dR);
    for (size_t q = 0; q < n2; q++) w->dKR1[q] = 2.0 * p->one_m_fR * w->d1[q] + w->dR[q];
    /* term 1: calc_λ_∂fKR1c∂uc! */
    for (int j = 0; j < m; j++)
        for (int t = 0; t < nt; t++) {
            cplx s = 0.0;
            for (int i = 0; i < m; i++)
                s += w->lt[(size_t)nt * i + t] * w->dKR1[(size_t)nt * (i + m * j) + t];
            w->sres[(size_t)nt * j + t] = s;
        }
    fft_cols(&w->pl, w->sres, m, 1);
    for (size_t q = 0; q < n1; q++) w->t1[q] = I * w->em[q] * w->sres[q];
    /* term 2: calc_λc_∂fK∂uc! */
    for (int j = 0; j < m; j++)
        for (int t = 0; t < nt; t++) {
            cplx s = 0.0;
            for (int i = 0; i < m; i++)
                s += w->lwc[(size_t)nt * i + t] * w->d2[(size_t)nt * (i + m * j) + t];
            w->sres[(size_t)nt * j + t] = s;
        }
    fft_cols(&w->pl, w->sres, m, 1);
    for (size_t q = 0; q < n1; q++) w->t2[q] = -I * (double)nt * w->em[q] * w->sres[q];
    /* term 3: calc_λ_∂fR2c∂uc! */
    calc_gamma_a_b(p, w->lt, w->utc, w->gab);
    fft_cols(&w->pl, w->gab, mm, 0);
    for (int c = 0; c < mm; c++)
        for (int t = 0; t < nt; t++)
            w->gab[(size_t)nt * c + t] *= conj(hR[t]) * w->sigma[t];
    fft_cols(&w->pl, w->gab, mm, 0);
    for (int i = 0; i < m; i++)
        for (int t = 0; t < nt; t++) {
            cplx s = 0.0;
            for (int j = 0; j < m; j++)
                s += w->gab[(size_t)nt * (i + m * j) + t] * w->uwi[(size_t)nt * j + t];
            w->gout[(size_t)nt * i + t] = s;
        }
    fft_cols(&w->pl, w->gout, m, 0);
    for (size_t q = 0; q < n1; q++) w->t3[q] = I / (double)nt * w->em[q] * w->gout[q];
    /* term 4: calc_λc_∂fR∂uc! */
    calc_gamma_a_b(p, w->lwc, w->ut, w->gab2);
    fft_cols(&w->pl, w->gab2, mm, 1);
    for (int c = 0; c < mm; c++)
        for (int t = 0; t < nt; t++)
            w->gab2[(size_t)nt * c + t] *= hR[t] * w->sigma[t];
    fft_cols(&w->pl, w->gab2, mm, 0);
    for (int i = 0; i < m; i++)
        for (int t = 0; t < nt; t++) {
            cplx s = 0.0;
            for (int j = 0; j < m; j++)
                s += w->gab2[(size_t)nt * (i + m * j) + t] * w->ut[(size_t)nt * j + t];
            w->gout[(size_t)nt * i + t] = s;
        }
    fft_cols(&w->pl, w->gout, m, 1);
    for (size_t q = 0; q < n1; q++) w->t4[q] = -I * (double)nt * w->em[q] * w->gout[q];
    for (size_t q = 0; q < n1; q++)
        dlam[q] = w->t1[q] + p->one_m_fR * w->t2[q] + w->t3[q] + w->t4[q];
}

/* ------------------------------------------------------------------------ */
/* Validation                                                                */
/* ------------------------------------------------------------------------ */

static int problem_valid(const orc_problem *p) {
    if (!p || p->nt < 4 || (p->nt & (p->nt - 1)) || p->m < 1) return 0;
    if (!p->D || !p->gamma || !p->hR || !p->selfsteep) return 0;
    if (!(p->L > 0) || !isfinite(p->L)) return 0;
    if (!(p->reltol > 0) || !isfinite(p->reltol)) return 0;
    if (!(p->abstol > 0) || !isfinite(p->abstol)) return 0;
    size_t m4 = (size_t)p->m * p->m * p->m * p->m;
    for (size_t i = 0; i < m4; i++)
        if (!isfinite(p->gamma[i])) return 0;
    return 1;
}

/* _adjoint_gamma_symmetric, sensitivity_disp_mmf.jl:103-112 */
static int approx_eq(double a, double b, double atol) {
    double d = fabs(a - b);
    double mx = fabs(a) > fabs(b) ? fabs(a) : fabs(b);
    return d <= (atol > 1e-12 * mx ? atol : 1e-12 * mx);
}

static int gamma_symmetric(const orc_problem *p) {
    int m = p->m;
    double mx = 0.0;
    size_t m4 = (size_t)m * m * m * m;
    for (size_t i = 0; i < m4; i++)
        if (fabs(p->gamma[i]) > mx) mx = fabs(p->gamma[i]);
    double tol = 1e-12 * (mx > 1.0 ? mx : 1.0);
    for (int l = 0; l < m; l++)
        for (int k = 0; k < m; k++)
            for (int j = 0; j < m; j++)
                for (int i = 0; i < m; i++) {
                    double v = G4(p->gamma, m, i, j, k, l);
                    if (!approx_eq(v, G4(p->gamma, m, j, i, k, l), tol)) return 0;
                    if (!approx_eq(v, G4(p->gamma, m, i, k, j, l), tol)) return 0;
                    if (!approx_eq(v, G4(p->gamma, m, i, j, l, k), tol)) return 0;
                }
    return 1;
}

int orc_rhs_forward(const orc_problem *p, double z, const orc_c64 *u, orc_c64 *du) {
    if (!problem_valid(p)) return ORC_EINVAL;
    workspace w;
    if (ws_init(&w, p, 0)) return ORC_ENOMEM;
    rhs_forward_ws(&w, z, (const cplx *)u, (cplx *)du);
    ws_free(&w);
    return ORC_OK;
}

int orc_rhs_adjoint(const orc_problem *p, double z, const orc_c64 *lam,
                    const orc_c64 *u_fwd, orc_c64 *dlam) {
    if (!problem_valid(p)) return ORC_EINVAL;
    workspace w;
    if (ws_init(&w, p, 1)) return ORC_ENOMEM;
    rhs_adjoint_ws(&w, z, (const cplx *)lam, (const cplx *)u_fwd, (cplx *)dlam);
    ws_free(&w);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Tsit5 (Tsitouras 2011) with OrdinaryDiffEq's default PI controller       */
/* ------------------------------------------------------------------------ */

static const double T5_c[7] = {0.0, 0.161, 0.327, 0.9, 0.9800255409045097, 1.0, 1.0};
static const double T5_a[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {0.161, 0, 0, 0, 0, 0},
    {-0.008480655492356989, 0.335480655492357, 0, 0, 0, 0},
    {2.897153057105493, -6.359448489975075, 4.3622954328695815, 0, 0, 0},
    {5.325864828439257, -11.748883564062828, 7.4955393428898365, -0.09249506636175525, 0, 0},
    {5.86145544294642, -12.92096931784711, 8.159367898576159, -0.071584973281401,
     -0.028269050394068383, 0},
    {0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081,
     2.324710524099774}};
static const double T5_btilde[7] = {-0.00178001105222577714, -0.0008164344596567469,
                                    0.007880878010261995,    -0.1447110071732629,
                                    0.5823571654525552,      -0.45808210592918697,
                                    0.015151515151515152};
/* free interpolant: b_i(θ) = Σ_{p=1..4} R[i][p-1] θ^p */
static const double T5_r[7][4] = {
    {1.0, -2.763706197274826, 2.9132554618219126, -1.0530884977290216},
    {0.0, 0.13169999999999998, -0.2234, 0.1017},
    {0.0, 3.9302962368947516, -5.941033872131505, 2.490627285651253},
    {0.0, -12.411077166933676, 30.33818863028232, -16.548102889244902},
    {0.0, 37.50931341651104, -88.1789048947664, 47.37952196281928},
    {0.0, -27.896526289197286, 65.09189467479366, -34.87065786149661},
    {0.0, 1.5, -4.0, 2.5}};

int orc_tsit5_order_residuals(double th, double *res, int nres) {
    /* b_i(θ) order conditions up to 4th order and the step tableau's 5th-order
     * quadrature conditions. */
    double b[7];
    for (int i = 0; i < 7; i++) {
        double s = 0.0, tp = th;
        for (int q = 0; q < 4; q++) {
            s += T5_r[i][q] * tp;
            tp *= th;
        }
        b[i] = s;
    }
    double ac[7];
    for (int i = 0; i < 7; i++) {
        double s = 0.0;
        for (int j = 0; j < i; j++) s += T5_a[i][j] * T5_c[j];
        ac[i] = s;
    }
    double r[16];
    int n = 0;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0, s6 = 0, s7 = 0;
    for (int i = 0; i < 7; i++) {
        s0 += b[i];
        s1 += b[i] * T5_c[i];
        s2 += b[i] * T5_c[i] * T5_c[i];
        s3 += b[i] * ac[i];
        s4 += b[i] * T5_c[i] * T5_c[i] * T5_c[i];
        s5 += b[i] * T5_c[i] * ac[i];
        double aac = 0.0, acc = 0.0;
        for (int j = 0; j < i; j++) {
            aac += T5_a[i][j] * ac[j];
            acc += T5_a[i][j] * T5_c[j] * T5_c[j];
        }
        s6 += b[i] * aac;
        s7 += b[i] * acc;
    }
    r[n++] = s0 - th;
    r[n++] = s1 - th * th / 2.0;
    r[n++] = s2 - th * th * th / 3.0;
    r[n++] = s3 - th * th * th / 6.0;
    r[n++] = s4 - pow(th, 4) / 4.0;
    r[n++] = s5 - pow(th, 4) / 8.0;
    r[n++] = s6 - pow(th, 4) / 24.0;
    r[n++] = s7 - pow(th, 4) / 12.0;
    /* row sums a_ij = c_i and b̃ sums to zero */
    double rs = 0.0, bt = 0.0;
    for (int i = 1; i < 7; i++) {
        double s = 0.0;
        for (int j = 0; j < i; j++) s += T5_a[i][j];
        rs += fabs(s - T5_c[i]);
    }
    for (int i = 0; i < 7; i++) bt += T5_btilde[i];
    r[n++] = rs;
    r[n++] = bt;
    /* interpolant at θ=1 reproduces the step weights (row 7 of a) */
    double e1 = 0.0;
    for (int i = 0; i < 7; i++) {
        double s = 0.0;
        for (int q = 0; q < 4; q++) s += T5_r[i][q];
        e1 += fabs(s - (i < 6 ? T5_a[6][i] : 0.0));
    }
    r[n++] = e1;
    for (int i = 0; i < n && i < nres; i++) res[i] = r[i];
    return n;
}

struct orc_dense {
    int nt, m;
    long nsteps, cap;
    double *t, *dt;     /* per step */
    cplx *coef;         /* per step: 5 vectors (u_n, c1..c4), each nt*m */
};

static int dense_push(orc_dense *d, double t, double dt, const cplx *u, cplx *const *k) {
    size_t n1 = (size_t)d->nt * d->m;
    if (d->nsteps == d->cap) {
        long nc = d->cap ? d->cap * 2 : 64;
        double *tt = (double *)realloc(d->t, sizeof(double) * nc);
        if (!tt) return -1;
        d->t = tt;
        double *dd = (double *)realloc(d->dt, sizeof(double) * nc);
        if (!dd) return -1;
        d->dt = dd;
        cplx *cc = (cplx *)realloc(d->coef, sizeof(cplx) * n1 * 5 * (size_t)nc);
        if (!cc) return -1;
        d->coef = cc;
        d->cap = nc;
    }
    cplx *c = d->coef + (size_t)d->nsteps * 5 * n1;
    memcpy(c, u, sizeof(cplx) * n1);
    for (int q = 0; q < 4; q++) {
        cplx *cq = c + (size_t)(q + 1) * n1;
        for (size_t x = 0; x < n1; x++) {
            cplx s = 0.0;
            for (int i = 0; i < 7; i++)
                if (T5_r[i][q] != 0.0) s += T5_r[i][q] * k[i][x];
            cq[x] = s;
        }
    }
    d->t[d->nsteps] = t;
    d->dt[d->nsteps] = dt;
    d->nsteps++;
    return 0;
}

long orc_dense_steps(const orc_dense *d) { return d ? d->nsteps : 0; }

int orc_dense_times(const orc_dense *d, double *t_out) {
    if (!d) return ORC_EINVAL;
    for (long s = 0; s < d->nsteps; s++) t_out[s] = d->t[s];
    if (d->nsteps > 0) t_out[d->nsteps] = d->t[d->nsteps - 1] + d->dt[d->nsteps - 1];
    return ORC_OK;
}

int orc_dense_eval(const orc_dense *d, double z, orc_c64 *out) {
    if (!d || d->nsteps == 0) return ORC_EINVAL;
    size_t n1 = (size_t)d->nt * d->m;
    /* interval s with t_s <= z <= t_s + dt_s (forward direction) */
    long lo = 0, hi = d->nsteps - 1;
    while (lo < hi) {
        long mid = (lo + hi + 1) / 2;
        if (d->t[mid] <= z) lo = mid;
        else hi = mid - 1;
    }
    long s = lo;
    const cplx *c = d->coef + (size_t)s * 5 * n1;
    double dt = d->dt[s];
    double th = (z - d->t[s]) / dt;
    double th2 = th * th, th3 = th2 * th, th4 = th3 * th;
    cplx *o = (cplx *)out;
    for (size_t x = 0; x < n1; x++)
        o[x] = c[x] + dt * (th * c[n1 + x] + th2 * c[2 * n1 + x] + th3 * c[3 * n1 + x] +
                            th4 * c[4 * n1 + x]);
    return ORC_OK;
}

void orc_dense_free(orc_dense *d) {
    if (!d) return;
    free(d->t);
    free(d->dt);
    free(d->coef);
    free(d);
}

typedef void (*rhs_fn)(void *ctx, double t, const cplx *u, cplx *du);

static double rms_norm_scaled(const cplx *x, const double *sk, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) {
        double a = cabs(x[i]) / sk[i];
        s += a * a;
    }
    return sqrt(s / (double)(n > 0 ? n : 1));
}

/* Hairer-style initial step (OrdinaryDiffEqCore ode_determine_initdt). */
static double initdt(rhs_fn f, void *ctx, size_t n, const cplx *u0, double t0, double tdir,
                     double dtmax, double reltol, double abstol, cplx *f0, cplx *f1, cplx *u1,
                     double *sk, long *nf, double dtmin) {
    for (size_t i = 0; i < n; i++) sk[i] = abstol + cabs(u0[i]) * reltol;
    f(ctx, t0, u0, f0);
    (*nf)++;
    double d0 = 0.0, d1 = 0.0;
    for (size_t i = 0; i < n; i++) {
        double a = cabs(u0[i]) / sk[i], b = cabs(f0[i]) / sk[i];
        d0 += a * a;
        d1 += b * b;
    }
    d0 = sqrt(d0 / (double)n);
    d1 = sqrt(d1 / (double)n);
    if (isnan(d1)) return tdir * dtmin;
    double smalldt = 1e-6;
    double dt0 = (d0 < 1e-5 || d1 < 1e-5) ? smalldt : (d0 / d1) / 100.0;
    if (dt0 > dtmax) dt0 = dtmax;
    if (dt0 < 10.0 * 2.220446049250313e-16) return tdir * (smalldt > dtmin ? smalldt : dtmin);
    for (size_t i = 0; i < n; i++) u1[i] = u0[i] + tdir * dt0 * f0[i];
    f(ctx, t0 + tdir * dt0, u1, f1);
    (*nf)++;
    double d2 = 0.0;
    int same = 1;
    for (size_t i = 0; i < n; i++) {
        if (f0[i] != f1[i]) same = 0;
        double a = cabs(f1[i] - f0[i]) / sk[i];
        d2 += a * a;
    }
    if (same && n > 0) return tdir * (dtmin > 100.0 * dt0 ? dtmin : 100.0 * dt0);
    d2 = sqrt(d2 / (double)n) / dt0;
    double mx = d1 > d2 ? d1 : d2;
    double dt1;
    if (mx <= 1e-15) {
        dt1 = dt0 * 1e-3;
        if (dt1 < 1e-6) dt1 = 1e-6;
    } else {
        dt1 = pow(10.0, -(2.0 + log10(mx)) / 5.0);
    }
    double r = 100.0 * dt0;
    if (dt1 < r) r = dt1;
    if (dtmax < r) r = dtmax;
    if (dtmin > r) r = dtmin;
    return tdir * r;
}

static int tsit5_solve(rhs_fn f, void *ctx, size_t n, const cplx *u0, double t0, double tf,
                       double reltol, double abstol, cplx *u_out, orc_stats *st,
                       orc_dense *dense) {
    const double beta1 = 7.0 / 50.0, beta2 = 2.0 / 25.0, gam = 0.9;
    const double qmin = 0.2, qmax = 10.0, qoldinit = 1e-4;
    const long maxiters = 100000;
    double tdir = tf > t0 ? 1.0 : -1.0;
    double span = fabs(tf - t0);
    double dtmax = span;
    double dtmin = 2.220446049250313e-16 * (fabs(t0) > fabs(tf) ? fabs(t0) : fabs(tf));
    if (dtmin <= 0) dtmin = 1e-300;
    cplx *buf = (cplx *)malloc(sizeof(cplx) * n * 11);
    double *sk = (double *)malloc(sizeof(double) * n);
    if (!buf || !sk) {
        free(buf);
        free(sk);
        return ORC_ENOMEM;
    }
    cplx *k[7];
    for (int i = 0; i < 7; i++) k[i] = buf + (size_t)i * n;
    cplx *u = buf + 7 * n, *unew = buf + 8 * n, *tmp = buf + 9 * n, *utilde = buf + 10 * n;
    memcpy(u, u0, sizeof(cplx) * n);
    st->naccept = st->nreject = st->nf = 0;
    st->retcode = ORC_OK;
    double dt = initdt(f, ctx, n, u0, t0, tdir, dtmax, reltol, abstol, k[0], k[1], tmp, sk,
                       &st->nf, dtmin);
    double t = t0;
    f(ctx, t, u, k[0]);
    st->nf++;
    double qold = qoldinit;
    long iter = 0;
    int rc = ORC_OK;
    while (tdir * t < tdir * tf) {
        if (++iter > maxiters) {
            rc = ORC_MAXITERS;
            break;
        }
        /* fix_dt_at_bounds!, modify_dt_for_tstops! */
        double adt = fabs(dt);
        if (adt > dtmax) adt = dtmax;
        if (adt < dtmin) adt = dtmin;
        double rem = fabs(tf - t);
        if (adt > rem) adt = rem;
        dt = tdir * adt;
        if (adt <= dtmin && rem > dtmin) {
            rc = ORC_DT_UNDERFLOW;
            break;
        }
        for (int s = 1; s < 7; s++) {
            for (size_t i = 0; i < n; i++) {
                cplx acc = 0.0;
                for (int j = 0; j < s; j++) acc += T5_a[s][j] * k[j][i];
                tmp[i] = u[i] + dt * acc;
            }
            if (s == 6) memcpy(unew, tmp, sizeof(cplx) * n);
            f(ctx, t + T5_c[s] * dt, tmp, k[s]);
            st->nf++;
        }
        for (size_t i = 0; i < n; i++) {
            cplx acc = 0.0;
            for (int j = 0; j < 7; j++) acc += T5_btilde[j] * k[j][i];
            utilde[i] = dt * acc;
            double a = cabs(u[i]), b = cabs(unew[i]);
            sk[i] = abstol + (a > b ? a : b) * reltol;
        }
        double EEst = rms_norm_scaled(utilde, sk, n);
        if (!isfinite(EEst)) {
            rc = ORC_NONFINITE;
            break;
        }
        double q11 = 0.0, q;
        if (EEst == 0.0) {
            q = 1.0 / qmax;
        } else {
            q11 = pow(EEst, beta1);
            q = q11 / pow(qold, beta2);
            q = q / gam;
            if (q > 1.0 / qmin) q = 1.0 / qmin;
            if (q < 1.0 / qmax) q = 1.0 / qmax;
        }
        if (EEst <= 1.0) {
            st->naccept++;
            if (dense && dense_push(dense, t, dt, u, k)) {
                rc = ORC_ENOMEM;
                break;
            }
            double ttmp = t + dt;
            /* fixed_t_for_floatingpoint_error!: snap within 100 eps of the tstop */
            double mxt = t > tf ? t : tf;
            if (fabs(ttmp - tf) < 100.0 * 2.220446049250313e-16 * fabs(mxt)) ttmp = tf;
            t = ttmp;
            memcpy(u, unew, sizeof(cplx) * n);
            memcpy(k[0], k[6], sizeof(cplx) * n);
            qold = EEst > qoldinit ? EEst : qoldinit;
            double dtnew = fabs(dt) / q; /* qsteady_min = qsteady_max = 1 */
            if (q == 1.0) dtnew = fabs(dt);
            if (dtnew > dtmax) dtnew = dtmax;
            if (dtnew < dtmin) dtnew = dtmin;
            dt = tdir * dtnew;
            for (size_t i = 0; i < n; i++)
                if (!isfinite(creal(u[i])) || !isfinite(cimag(u[i]))) {
                    rc = ORC_NONFINITE;
                    break;
                }
            if (rc) break;
        } else {
            st->nreject++;
            double den = q11 / gam;
            if (den > 1.0 / qmin) den = 1.0 / qmin;
            dt = dt / den;
        }
    }
    st->retcode = rc;
    st->z_end = t;
    if (u_out) memcpy(u_out, u, sizeof(cplx) * n);
    free(buf);
    free(sk);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Pump-gain propagation (simulate_disp_gain_mmf.jl, gain_simulation/gain.jl) */
/* ------------------------------------------------------------------------ */

/* compute_gain: g(w) per bin into gw, returns the pump gain g_P.  The YDFA
 * branch is calculate_gain_YDFA (gain.jl:150-166) on the PSD of
 * psd_from_uw (gain.jl:122-127): the sums over bins do not depend on the bin
 * order, so everything stays in FFT order. */
static double gain_profile(const orc_gain *g, int nt, const cplx *uw, double Pp, double *gw) {
    if (g->kind == 0) {
        for (int b = 0; b < nt; b++) gw[b] = g->g_const;
        return -1.0;
    }
    double W12 = 0.0, W21 = 0.0;
    for (int b = 0; b < nt; b++) {
        const double a = cabs(uw[b]);
        const double Ps = a * a * g->psd_scale;
        W12 += g->gamma_s * g->sigma_as[b] * Ps * g->df / (g->h_nu_s[b] * g->area);
        W21 += g->gamma_s * g->sigma_es[b] * Ps * g->df / (g->h_nu_s[b] * g->area);
    }
    const double R12 = g->gamma_p * g->sigma_ap * Pp / (g->h_nu_p * g->area);
    const double R21 = g->gamma_p * g->sigma_ep * Pp / (g->h_nu_p * g->area);
    const double n2 = (R12 + W12) / (R12 + R21 + W12 + W21 + 1.0 / g->tau21);
    const double n1 = 1.0 - n2;
    for (int b = 0; b < nt; b++)
        gw[b] = g->gamma_s * (g->sigma_es[b] * n2 - g->sigma_as[b] * n1) * g->rho;
    return g->gamma_p * (g->sigma_ep * n2 - g->sigma_ap * n1) * g->rho;
}

typedef struct {
    workspace w;
    const orc_gain *g;
    cplx *uw;
    double *gw;
} gain_ctx;

static void gain_rhs_cb(void *ctx, double z, const cplx *u, cplx *du) {
    gain_ctx *c = (gain_ctx *)ctx;
    const orc_problem *p = c->w.p;
    const int nt = p->nt;
    const cplx *ut = u + 1;
    /* compute_gain takes the lab-frame field e^{iDz} u~ and the pump power */
    for (int b = 0; b < nt; b++) {
        const double a = p->D[b] * z;
        c->uw[b] = (cos(a) + I * sin(a)) * ut[b];
    }
    const double gP = gain_profile(c->g, nt, c->uw, creal(u[0]), c->gw);
    rhs_forward_ws(&c->w, z, ut, du + 1);
    for (int b = 0; b < nt; b++) du[1 + b] += 0.5 * c->gw[b] * ut[b];
    du[0] = gP * u[0];
}

static int gain_ctx_init(gain_ctx *c, const orc_problem *p, const orc_gain *g) {
    memset(c, 0, sizeof(*c));
    if (!problem_valid(p) || p->m != 1 || !g || (g->kind != 0 && g->kind != 1)) return ORC_EINVAL;
    if (g->kind == 1 && (!g->sigma_as || !g->sigma_es || !g->h_nu_s)) return ORC_EINVAL;
    if (ws_init(&c->w, p, 0)) return ORC_ENOMEM;
    c->g = g;
    c->uw = (cplx *)malloc(sizeof(cplx) * p->nt);
    c->gw = (double *)malloc(sizeof(double) * p->nt);
    if (!c->uw || !c->gw) return ORC_ENOMEM;
    return ORC_OK;
}

static void gain_ctx_free(gain_ctx *c) {
    ws_free(&c->w);
    free(c->uw);
    free(c->gw);
}

int orc_rhs_gain(const orc_problem *p, const orc_gain *g, double z, const orc_c64 *state,
                 orc_c64 *dstate) {
    gain_ctx c;
    int rc = gain_ctx_init(&c, p, g);
    if (rc == ORC_OK) gain_rhs_cb(&c, z, (const cplx *)state, (cplx *)dstate);
    gain_ctx_free(&c);
    return rc;
}

int orc_forward_gain(const orc_problem *p, const orc_gain *g, double pump0,
                     const orc_c64 *u0, int nsave, const double *zsave, orc_c64 *out,
                     double *pump_out, orc_stats *st) {
    gain_ctx c;
    int rc = gain_ctx_init(&c, p, g);
    const int nt = p ? p->nt : 0;
    const size_t n = (size_t)nt + 1;
    if (rc == ORC_OK && (nsave < 0 || (nsave > 0 && (!zsave || !out || !pump_out))))
        rc = ORC_EINVAL;
    cplx *s0 = rc == ORC_OK ? (cplx *)malloc(sizeof(cplx) * n) : NULL;
    cplx *sL = rc == ORC_OK ? (cplx *)malloc(sizeof(cplx) * n) : NULL;
    cplx *sz = rc == ORC_OK ? (cplx *)malloc(sizeof(cplx) * n) : NULL;
    orc_dense *d = rc == ORC_OK ? (orc_dense *)calloc(1, sizeof(orc_dense)) : NULL;
    if (rc == ORC_OK && (!s0 || !sL || !sz || !d)) rc = ORC_ENOMEM;
    orc_stats local;
    if (!st) st = &local;
    if (rc == ORC_OK) {
        d->nt = nt + 1;  /* the dense output of the whole state [P; u~] */
        d->m = 1;
        /* u0 = vcat(Pp0, u_w0) (simulate_disp_gain_mmf.jl:218-219) */
        s0[0] = pump0;
        for (int b = 0; b < nt; b++) {
            s0[1 + b] = u0[b].re + I * u0[b].im;
            if (!isfinite(u0[b].re) || !isfinite(u0[b].im)) rc = ORC_NONFINITE;
        }
    }
    if (rc == ORC_OK)
        rc = tsit5_solve(gain_rhs_cb, &c, n, s0, 0.0, p->L, p->reltol, p->abstol, sL, st, d);
    if (rc == ORC_OK && st->z_end != p->L) rc = ORC_EINVAL;
    for (int k = 0; rc == ORC_OK && k < nsave; k++) {
        const double z = zsave[k];
        if (!(z >= 0.0 && z <= p->L)) {
            rc = ORC_EINVAL;
            break;
        }
        if (z == 0.0) memcpy(sz, s0, sizeof(cplx) * n);
        else if (z == p->L) memcpy(sz, sL, sizeof(cplx) * n);
        else orc_dense_eval(d, z, (orc_c64 *)sz);
        pump_out[k] = creal(sz[0]);
        for (int b = 0; b < nt; b++) {
            const double a = p->D[b] * z;
            const cplx y = (cos(a) + I * sin(a)) * sz[1 + b];
            out[(size_t)k * nt + b].re = creal(y);
            out[(size_t)k * nt + b].im = cimag(y);
        }
    }
    free(s0);
    free(sL);
    free(sz);
    orc_dense_free(d);
    gain_ctx_free(&c);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Drivers                                                                   */
/* ------------------------------------------------------------------------ */

static void fwd_rhs_cb(void *ctx, double t, const cplx *u, cplx *du) {
    rhs_forward_ws((workspace *)ctx, t, u, du);
}

int orc_forward(const orc_problem *p, const orc_c64 *u0, int nsave, const double *zsave,
                orc_c64 *out, orc_stats *st, orc_dense **dense_out) {
    if (!problem_valid(p)) return ORC_EINVAL;
    size_t n1 = (size_t)p->nt * p->m;
    for (size_t i = 0; i < n1; i++)
        if (!isfinite(u0[i].re) || !isfinite(u0[i].im)) return ORC_NONFINITE;
    workspace w;
    if (ws_init(&w, p, 0)) return ORC_ENOMEM;
    orc_dense *d = (orc_dense *)calloc(1, sizeof(orc_dense));
    if (!d) {
        ws_free(&w);
        return ORC_ENOMEM;
    }
    d->nt = p->nt;
    d->m = p->m;
    cplx *uL = (cplx *)malloc(sizeof(cplx) * n1);
    orc_stats local;
    if (!st) st = &local;
    int rc = tsit5_solve(fwd_rhs_cb, &w, n1, (const cplx *)u0, 0.0, p->L, p->reltol, p->abstol,
                         uL, st, d);
    if (rc == ORC_OK && st->z_end != p->L) rc = ORC_EINVAL;
    if (rc == ORC_OK && out) {
        cplx *o = (cplx *)out;
        for (int s = 0; s < nsave; s++) {
            double z = zsave[s];
            cplx *os = o + (size_t)s * n1;
            if (z == 0.0) memcpy(os, u0, sizeof(cplx) * n1);
            else if (z == p->L) memcpy(os, uL, sizeof(cplx) * n1);
            else orc_dense_eval(d, z, (orc_c64 *)os);
            for (size_t i = 0; i < n1; i++) {
                double a = p->D[i] * z;
                os[i] = (cos(a) + I * sin(a)) * os[i];
            }
        }
    }
    free(uL);
    ws_free(&w);
    if (rc == ORC_OK && dense_out) *dense_out = d;
    else orc_dense_free(d);
    return rc;
}

typedef struct {
    workspace w;
    const orc_dense *fwd;
} adj_ctx;

static void adj_rhs_cb(void *ctx, double t, const cplx *u, cplx *du) {
    adj_ctx *a = (adj_ctx *)ctx;
    orc_dense_eval(a->fwd, t, (orc_c64 *)a->w.ufwd);
    rhs_adjoint_ws(&a->w, t, u, a->w.ufwd, du);
}

int orc_adjoint(const orc_problem *p, const orc_dense *fwd, const orc_c64 *lambdaL,
                orc_c64 *lambda0, orc_stats *st) {
    if (!problem_valid(p) || !fwd) return ORC_EINVAL;
    if (!gamma_symmetric(p)) return ORC_NONSYMMETRIC;
    size_t n1 = (size_t)p->nt * p->m;
    cplx *lt = (cplx *)malloc(sizeof(cplx) * n1);
    if (!lt) return ORC_ENOMEM;
    double scale = 0.0;
    for (size_t i = 0; i < n1; i++) {
        double a = -p->D[i] * p->L;
        lt[i] = (cos(a) + I * sin(a)) * (*(const cplx *)&lambdaL[i]);
        if (!isfinite(creal(lt[i])) || !isfinite(cimag(lt[i]))) {
            free(lt);
            return ORC_NONFINITE;
        }
        double ab = cabs(lt[i]);
        if (ab > scale) scale = ab;
    }
    double abstol = scale == 0.0 ? p->abstol : p->abstol * scale;
    adj_ctx a;
    a.fwd = fwd;
    if (ws_init(&a.w, p, 1)) {
        free(lt);
        return ORC_ENOMEM;
    }
    orc_stats local;
    if (!st) st = &local;
    int rc = tsit5_solve(adj_rhs_cb, &a, n1, lt, p->L, 0.0, p->reltol, abstol,
                         (cplx *)lambda0, st, NULL);
    ws_free(&a.w);
    free(lt);
    return rc;
}

int orc_rk4_scalar(const orc_problem *p, const orc_c64 *u0, int steps, orc_c64 *out) {
    if (!problem_valid(p) || p->m != 1 || steps <= 0) return ORC_EINVAL;
    int nt = p->nt;
    fft_plan pl;
    if (plan_init(&pl, nt)) return ORC_ENOMEM;
    cplx *buf = (cplx *)malloc(sizeof(cplx) * nt * 9);
    if (!buf) {
        plan_free(&pl);
        return ORC_ENOMEM;
    }
    cplx *u = buf, *k1 = buf + nt, *k2 = buf + 2 * nt, *k3 = buf + 3 * nt, *k4 = buf + 4 * nt;
    cplx *tmp = buf + 5 * nt, *tf = buf + 6 * nt, *ni = buf + 7 * nt, *sh = buf + 8 * nt;
    const cplx *hR = (const cplx *)p->hR;
    double gamma = p->gamma[0];
    memcpy(u, u0, sizeof(cplx) * nt);
    /* rhs(z, ũ), scalar_crosscheck.jl:38-48 */
#define SCALAR_RHS(z, in, outv)                                                     \
    do {                                                                            \
        for (int t = 0; t < nt; t++) {                                              \
            double a = p->D[t] * (z);                                               \
            tf[t] = (cos(a) + I * sin(a)) * (in)[t];                                \
        }                                                                           \
        fft_1d(&pl, tf, 0);                                                         \
        for (int t = 0; t < nt; t++) ni[t] = gamma * (creal(tf[t]) * creal(tf[t]) + \
                                                      cimag(tf[t]) * cimag(tf[t])); \
        fft_1d(&pl, ni, 0);                                                         \
        for (int t = 0; t < nt; t++) ni[t] *= hR[t];                                \
        fft_1d(&pl, ni, 1);                                                         \
        fftshift_cols(ni, sh, nt, 1);                                               \
        for (int t = 0; t < nt; t++) {                                              \
            double inten = gamma * (creal(tf[t]) * creal(tf[t]) +                   \
                                    cimag(tf[t]) * cimag(tf[t]));                   \
            ni[t] = (p->one_m_fR * inten + creal(sh[t])) * tf[t];                   \
        }                                                                           \
        fft_1d(&pl, ni, 1);                                                         \
        for (int t = 0; t < nt; t++) {                                              \
            double a = -p->D[t] * (z);                                              \
            (outv)[t] = I * (cos(a) + I * sin(a)) * (p->selfsteep[t] * ni[t]);      \
        }                                                                           \
    } while (0)
    double h = p->L / steps;
    for (int s = 0; s < steps; s++) {
        double z = s * h;
        SCALAR_RHS(z, u, k1);
        for (int t = 0; t < nt; t++) tmp[t] = u[t] + h / 2 * k1[t];
        SCALAR_RHS(z + h / 2, tmp, k2);
        for (int t = 0; t < nt; t++) tmp[t] = u[t] + h / 2 * k2[t];
        SCALAR_RHS(z + h / 2, tmp, k3);
        for (int t = 0; t < nt; t++) tmp[t] = u[t] + h * k3[t];
        SCALAR_RHS(z + h, tmp, k4);
        for (int t = 0; t < nt; t++) u[t] += h / 6 * (k1[t] + 2.0 * k2[t] + 2.0 * k3[t] + k4[t]);
    }
#undef SCALAR_RHS
    cplx *o = (cplx *)out;
    for (int t = 0; t < nt; t++) {
        double a = p->D[t] * p->L;
        o[t] = (cos(a) + I * sin(a)) * u[t];
    }
    free(buf);
    plan_free(&pl);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Batched band-objective phase gradient (CPU baseline)                     */
/* ------------------------------------------------------------------------ */

/* One problem: shaped launch (physics_models.jl:791-797), forward, band cost
 * and seed (physics_helpers.jl:222-232), adjoint, and the vector-phase
 * gradient 2 Re(conj(λ0) i u_shaped) summed over modes
 * (physics_models.jl:1042, :732-737). */
static int phase_gradient_one(const orc_problem *p, const orc_c64 *u0, const double *phase,
                              const unsigned char *mask, double *J, double *grad,
                              long *nsteps) {
    int nt = p->nt, m = p->m;
    size_t n1 = (size_t)nt * m;
    cplx *us = (cplx *)malloc(sizeof(cplx) * n1 * 3);
    if (!us) return ORC_ENOMEM;
    cplx *uL = us + n1, *lam = us + 2 * n1;
    for (int i = 0; i < m; i++)
        for (int t = 0; t < nt; t++) {
            size_t q = (size_t)nt * i + t;
            us[q] = (cos(phase[t]) + I * sin(phase[t])) * (*(const cplx *)&u0[q]);
        }
    double zs[1] = {p->L};
    orc_dense *d = NULL;
    orc_stats st;
    int rc = orc_forward(p, (const orc_c64 *)us, 1, zs, (orc_c64 *)uL, &st, &d);
    if (rc) {
        free(us);
        return rc;
    }
    long steps = st.naccept + st.nreject;
    double tot = 0.0, band = 0.0;
    for (int i = 0; i < m; i++)
        for (int t = 0; t < nt; t++) {
            double e = creal(uL[(size_t)nt * i + t]) * creal(uL[(size_t)nt * i + t]) +
                       cimag(uL[(size_t)nt * i + t]) * cimag(uL[(size_t)nt * i + t]);
            tot += e;
            if (mask[t]) band += e;
        }
    double cost = band / tot;
    for (int i = 0; i < m; i++)
        for (int t = 0; t < nt; t++) {
            size_t q = (size_t)nt * i + t;
            lam[q] = uL[q] * ((mask[t] ? 1.0 : 0.0) - cost) / tot;
        }
    rc = orc_adjoint(p, d, (const orc_c64 *)lam, (orc_c64 *)lam, &st);
    steps += st.naccept + st.nreject;
    orc_dense_free(d);
    if (rc) {
        free(us);
        return rc;
    }
    for (int t = 0; t < nt; t++) {
        double g = 0.0;
        for (int i = 0; i < m; i++) {
            size_t q = (size_t)nt * i + t;
            g += 2.0 * creal(conj(lam[q]) * (I * us[q]));
        }
        grad[t] = g;
    }
    *J = cost;
    if (nsteps) *nsteps = steps;
    free(us);
    return ORC_OK;
}

int orc_batch_phase_gradient(const orc_problem *p, const orc_c64 *u0, const double *phases,
                             int nprob, const unsigned char *mask, double *J, double *grad,
                             long *nsteps, int nthreads) {
    int failed = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : failed)
#endif
    for (int b = 0; b < nprob; b++) {
        long ns = 0;
        int rc = phase_gradient_one(p, u0, phases + (size_t)b * p->nt, mask, &J[b],
                                    grad + (size_t)b * p->nt, &ns);
        if (nsteps) nsteps[b] = ns;
        if (rc) failed++;
    }
    (void)nthreads;
    return failed;
}
