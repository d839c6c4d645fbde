/*
 * fl_oracle.h -- FP64 CPU restatement of FiberLab's GMMNLSE forward and
 * adjoint solvers.  TEST INFRASTRUCTURE ONLY: this library is the parity
 * checker for the CUDA path and the timed CPU baseline.  Nothing in the
 * product links or calls it.
 *
 * Array conventions follow the reference (Julia, column-major):
 *   field  (Nt, M)       element (t, i)      at t + Nt*i
 *   D      (Nt, M)       element (t, i)      at t + Nt*i        [rad/m]
 *   gamma  (M, M, M, M)  element (i,j,k,l)   at i + M*(j + M*(k + M*l))
 *   hR     (Nt,)         complex, FFT order
 *   selfsteep (Nt,)      fftshift(ωs/ω0), FFT order
 */
#ifndef FL_ORACLE_H
#define FL_ORACLE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double re, im;
} orc_c64;

typedef struct {
    int nt, m;
    const double *D;
    const double *gamma;
    const orc_c64 *hR;
    const double *selfsteep;
    double one_m_fR;
    double L;
    double reltol, abstol;
} orc_problem;

typedef struct {
    long naccept, nreject, nf;
    int retcode;          /* 0 ok, see ORC_* below */
    double z_end;
} orc_stats;

enum {
    ORC_OK = 0,
    ORC_EINVAL = 1,
    ORC_NONFINITE = 2,
    ORC_DT_UNDERFLOW = 3,
    ORC_MAXITERS = 4,
    ORC_ENOMEM = 5,
    ORC_NONSYMMETRIC = 6
};

typedef struct orc_dense orc_dense;

/* Unnormalised forward DFT (sign -1) and normalised inverse (1/N) along the
 * time axis of an (Nt, ncols) column-major complex array, in place. */
int orc_fft(orc_c64 *x, int nt, int ncols, int inverse);

/* One evaluation of the forward RHS (simulate_disp_mmf.jl:25-60). */
int orc_rhs_forward(const orc_problem *p, double z, const orc_c64 *u, orc_c64 *du);

/* One evaluation of the adjoint RHS (sensitivity_disp_mmf.jl:32-79) with
 * the forward field at z given directly (in place of the interpolant). */
int orc_rhs_adjoint(const orc_problem *p, double z, const orc_c64 *lam,
                    const orc_c64 *u_fwd, orc_c64 *dlam);

/* Forward Tsit5 solve 0 -> L (simulate_disp_mmf.jl:183-207,
 * propagation.jl:38-58, 89-123).  Writes lab-frame spectra cis(D z) u~(z) at
 * each of the nsave positions into out (Nt*M*nsave).  If dense_out is not
 * NULL the dense solution is kept for the adjoint. */
int orc_forward(const orc_problem *p, const orc_c64 *u0, int nsave,
                const double *zsave, orc_c64 *out, orc_stats *st,
                orc_dense **dense_out);

/* Interpolate the kept forward solution (interaction frame) at z. */
int orc_dense_eval(const orc_dense *d, double z, orc_c64 *u);
long orc_dense_steps(const orc_dense *d);
int orc_dense_times(const orc_dense *d, double *t_out);
void orc_dense_free(orc_dense *d);

/* Adjoint Tsit5 solve L -> 0 (sensitivity_disp_mmf.jl:309-332).  lambdaL is
 * the lab-frame terminal seed; lambda0 receives sol(0). */
int orc_adjoint(const orc_problem *p, const orc_dense *fwd,
                const orc_c64 *lambdaL, orc_c64 *lambda0, orc_stats *st);

/* Gain model of the pump-gain propagation (simulate_disp_gain_mmf.jl:68-102,
 * gain_simulation/gain.jl:25-166).  kind 0: constant gain g_const per metre
 * on every bin, pump gain -1 (the reference's placeholder); kind 1: the
 * Yb-doped fiber steady-state rate equations with the caller's cross
 * sections.  Per-bin arrays are in FFT bin order (the physical-order arrays
 * ifftshift-ed). */
typedef struct {
    int kind;
    double g_const;
    double gamma_p, sigma_ap, sigma_ep, h_nu_p;   /* pump overlap, cross sections [m^2], h nu_p [J] */
    double gamma_s, area, rho, tau21;             /* signal overlap, core area [m^2], ions [m^-3], lifetime [s] */
    double psd_scale;                             /* |u_w|^2 -> W/Hz: (Nt dt)^2 x repetition rate */
    double df;                                    /* bin width [Hz] */
    const double *sigma_as, *sigma_es;            /* Nt signal cross sections [m^2] */
    const double *h_nu_s;                         /* Nt photon energies [J] */
} orc_gain;

/* One evaluation of the pump-gain RHS (disp_gain_smf!,
 * simulate_disp_gain_mmf.jl:21-66) for M = 1: state (Nt + 1) complex values
 * [P_pump; u~]; dP/dz = g_P P, du~/dz = (disp_mmf! RHS) + g(w)/2 u~. */
int orc_rhs_gain(const orc_problem *p, const orc_gain *g, double z, const orc_c64 *state,
                 orc_c64 *dstate);

/* Pump-gain Tsit5 solve 0 -> L (solve_disp_gain_smf,
 * simulate_disp_gain_mmf.jl:204-239; the reference fixes reltol = 1e-5 and
 * keeps the default abstol: set them in p).  At each zsave position (sorted,
 * within [0, L]) out receives the lab-frame spectrum (Nt complex,
 * position-major) and pump_out the pump power, from the dense output. */
int orc_forward_gain(const orc_problem *p, const orc_gain *g, double pump0,
                     const orc_c64 *u0, int nsave, const double *zsave, orc_c64 *out,
                     double *pump_out, orc_stats *st);

/* Fixed-step RK4 scalar restatement (scalar_crosscheck.jl:38-67). */
int orc_rk4_scalar(const orc_problem *p, const orc_c64 *u0, int steps,
                   orc_c64 *out);

/* Tsit5 tableau self-check: fills order-condition residuals. */
int orc_tsit5_order_residuals(double theta, double *res, int nres);

/* Batched band-objective forward+adjoint phase gradients, one independent
 * problem per OpenMP thread (the CPU baseline).  phases: (Nt, nprob) launch
 * phase per problem shared over modes; mask: Nt bytes; J: nprob; grad:
 * (Nt, nprob).  Returns the number of failed problems. */
int orc_batch_phase_gradient(const orc_problem *p, const orc_c64 *u0,
                             const double *phases, int nprob,
                             const unsigned char *mask, double *J,
                             double *grad, long *nsteps, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
