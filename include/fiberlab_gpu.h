/*
 * fiberlab_gpu.h -- C-ABI of the B200 GMMNLSE stepper (forward propagation and
 * adjoint gradient of FiberLab's interaction-picture solver).
 *
 * The reference has no FFI layer: its boundary is two Julia functions,
 *   solve_disp_mmf(uω0, fiber, sim)            src/simulation/simulate_disp_mmf.jl:183
 *   solve_adjoint_disp_mmf(λωL, ũω, fiber, sim) src/simulation/sensitivity_disp_mmf.jl:309
 * and the callers built on them (propagate, src/fiberlab/propagation.jl:89;
 * the adjoint model's physical gradient, src/fiberlab/physics_models.jl:1033-1046).
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions
 *  - All functions return an int status (FL_OK = 0); no exception or longjmp
 *    crosses the ABI.  fl_last_error(ctx) returns the message of the last
 *    failure on that context.
 *  - Arrays are the reference's column-major Julia arrays, passed as plain
 *    host pointers: a field (Nt, M) of ComplexF64 is 2*Nt*M doubles with
 *    element (t, i) at [2*(t + Nt*i)] (re) and [2*(t + Nt*i) + 1] (im);
 *    D (Nt, M) is Nt*M doubles; gamma (M,M,M,M) is M^4 doubles with
 *    γ[i,j,k,l] at i + M*(j + M*(k + M*l)).
 *  - Host buffers are copied in and out; device buffers are owned by the
 *    context/problem.  Functions with the _device suffix take device pointers
 *    (already resident in HBM) instead.
 *  - One context per host thread: calls on one context are not thread-safe.
 *  - The GPU path is the only path: when no CUDA device or kernel image is
 *    available the calls fail with FL_ENODEV; there is no CPU fallback.
 */
#ifndef FIBERLAB_GPU_H
#define FIBERLAB_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (the solver codes mirror the reference's failure modes) */
#define FL_OK 0
#define FL_EINVAL 1          /* ArgumentError in the reference */
#define FL_NONFINITE 2       /* NaN/Inf in a stage or result */
#define FL_DT_UNDERFLOW 3    /* dt forced below floating-point resolution */
#define FL_MAXITERS 4        /* attempted-step limit reached */
#define FL_ENOMEM 5          /* device allocation failed */
#define FL_NONSYMMETRIC 6    /* adjoint needs a permutation-symmetric gamma */
#define FL_ENODEV 7          /* no usable CUDA device / kernel image */
#define FL_ECUDA 8           /* other CUDA runtime error */
#define FL_ECAPACITY 9       /* checkpoint/segment/step-log capacity exceeded */
#define FL_EUNSUPPORTED 10   /* shape not built (e.g. Nt outside 2^6..2^14) */
#define FL_OOM_ADMISSION 11  /* serving: request larger than the HBM budget */
#define FL_EBUSY 12          /* serving: request not finished */
#define FL_TIMEOUT 13        /* serving: wait limit reached */
#define FL_ECHECK 14         /* checked build (libfiberlab_gpu_checked.so): a solver state
                                index left its buffer's bounds; the slot stopped before
                                the access */

/* FP32 bulk, FP64 phase/norm/reductions/state.  The single-mode adjoint runs
 * in FP64; the multimode adjoint (M >= 6, Nt a multiple of 128) keeps λ and
 * its transforms in FP64 and takes the forward field's transform, pair
 * products and the per-point contractions at FP32 accuracy (3xTF32 tensor
 * cores, low-rank form of the overlap contraction where γ allows it). */
#define FL_PRECISION_FP32 0
#define FL_PRECISION_FP64 1  /* all arithmetic in FP64 */

typedef struct fl_ctx fl_ctx;
typedef struct fl_problem fl_problem;
typedef struct fl_server fl_server;

typedef struct {
    size_t hbm_budget_bytes;   /* 0: no limit beyond cudaMalloc */
    int checkpoints;           /* z-checkpoint slots K for the adjoint (power of 2, default 32) */
    int segment_steps;         /* dense-output steps kept (default 64).  A solve of at most
                                  segment_steps accepted steps keeps every step's interpolant
                                  during the forward and its adjoint recomputes nothing;
                                  longer solves recompute from the K checkpoints, replaying
                                  each checkpoint segment once per sub-segment of
                                  segment_steps steps (never failing for capacity), so K and
                                  segment_steps trade memory for recompute */
    int step_log;              /* accepted-step log capacity; 0 (default): max_iters entries,
                                  so the log never ends a solve the step limit admits */
    long max_iters;            /* attempted steps per integration (default 100000, as maxiters) */
} fl_ctx_opts;

/* Per-solve counters, mirroring destats.naccept/.nreject/.nf of the forward
 * ODESolution (src/fiberlab/propagation.jl:105-108) and of the adjoint. */
typedef struct {
    long naccept, nreject, nf;
    long adj_naccept, adj_nreject, adj_nf;
    int status;
    int checkpoints_used;
    double J;          /* objective value (band gradient calls) */
    double z_end;
    long recompute_steps;  /* forward steps recomputed by the adjoint from checkpoints
                              (0 when the forward kept every step's interpolant) */
} fl_stats;

/* Library version string and status names. */
const char *fl_version(void);
const char *fl_status_string(int status);

/* Context on one CUDA device. */
int fl_ctx_create(int device, const fl_ctx_opts *opts, fl_ctx **out);
int fl_ctx_destroy(fl_ctx *ctx);
const char *fl_last_error(const fl_ctx *ctx);
/* Kernel launches issued by this context since creation (evidence counter). */
long fl_ctx_launch_count(const fl_ctx *ctx);
/* Device time of the last public call on this context, measured with CUDA
 * events recorded on the context's stream: the whole call's GPU work and the
 * stepper kernel launches alone (milliseconds). */
int fl_ctx_timing(const fl_ctx *ctx, double *last_call_ms, double *last_kernel_ms);
/* Synchronise the context's stream. */
int fl_ctx_synchronize(fl_ctx *ctx);
/* Run every later call of this context on the caller's CUDA stream
 * (a cudaStream_t passed as void*; NULL returns to the context's private
 * stream; cudaStreamLegacy selects the legacy default stream).  Its work is
 * then ordered with the caller's own work on that stream: a device-buffer
 * entry point reads inputs that earlier work on the stream produced, without
 * a host synchronisation in between.  The entry points still synchronise the
 * stream before they return (they hand back statistics, and host-buffer
 * calls their outputs).  Work already queued on the previous stream is
 * waited for before the switch.  The reference's rule for concurrent solves
 * is one solve with its own state per thread
 * (agent-docs/current-agent-context/NUMERICS.md:35-37): here that is one
 * context per host thread, each on its own stream;
 * CUDA graphs the context captures are captured on its private stream and
 * launched on the current one. */
int fl_ctx_set_stream(fl_ctx *ctx, void *stream);
/* The stream the context's calls currently run on. */
void *fl_ctx_get_stream(const fl_ctx *ctx);

/* Upload one resolved problem: the tables get_p_disp_mmf builds from the
 * `fiber`/`sim` dictionaries (simulate_disp_mmf.jl:87-114,
 * sensitivity_disp_mmf.jl:237-283; required keys physics_models.jl:463-465).
 *   D        (Nt, M) dispersion Dω [rad/m]
 *   gamma    (M,M,M,M) real Kerr tensor [1/(W m)]
 *   hR       Nt complex (interleaved) Raman spectrum hRω, Hermitian
 *   selfsteep Nt: fftshift(ωs/ω0)
 * Validation mirrors the reference: real finite gamma
 * (simulate_disp_mmf.jl:62-67), Hermitian hR (physics_models.jl:438-449),
 * positive finite L, reltol, abstol (propagation.jl:41-44). */
int fl_problem_create(fl_ctx *ctx, int nt, int m, const double *D, const double *gamma,
                      const double *hR, const double *selfsteep, double one_m_fR, double L,
                      double reltol, double abstol, int precision, fl_problem **out);
int fl_problem_destroy(fl_problem *prob);

/* Terminal objective of the batched gradient entry points
 * (fl_phase_gradient_batch*, fl_mode_phase_gradient_batch*) and of the
 * problem's band-gradient server requests, computed on the device with its
 * seed λ(L) = ∂J/∂conj(u(L)).  Replaces the choice among the reference's
 * objective constructors raman_band_objective / fundamental_mode_objective /
 * worst_mode_objective / raman_peak_objective (physics_models.jl:851-932),
 * whose costs are physics_helpers.jl:222-302.  (temporal_width needs a
 * transform of the output; run it with fl_forward + fl_adjoint and a host
 * seed.)  The default is FL_OBJ_RAMAN_BAND; worst_mode_tau is the
 * log-sum-exp smoothness τ (reference default 50).  For M = 1 the
 * fundamental-mode and worst-mode objectives equal the band objective. */
#define FL_OBJ_RAMAN_BAND 0  /* mode-summed band fraction */
#define FL_OBJ_FUNDAMENTAL 1 /* band fraction of mode 1; seed zero on the others */
#define FL_OBJ_WORST_MODE 2  /* normalised log-sum-exp of the per-mode band fractions */
#define FL_OBJ_RAMAN_PEAK 3  /* strongest in-band bin (summed over modes) over the total */
int fl_problem_set_objective(fl_problem *prob, int objective, double worst_mode_tau);

/* Pump-gain single-mode forward solve 0 -> L.  Replaces solve_disp_gain_smf
 * (simulate_disp_gain_mmf.jl:204-239) with its right-hand side disp_gain_smf!
 * (:21-66): the state [P_pump; ũ], dP/dz = g_P P, and disp_mmf!'s derivative
 * plus g(ω) ũ / 2.  The gain is constant (FL_GAIN_CONSTANT: g_const per metre
 * on every bin, g_P = -1, the reference's placeholder, :74-78) or the
 * Yb-doped fiber steady-state rate equations (FL_GAIN_YDFA:
 * calculate_gain_YDFA, gain_simulation/gain.jl:150-166, on the PSD
 * |u_ω|² psd_scale of psd_from_uω, :122-127), whose per-bin arrays are in FFT
 * bin order (the reference's physical-order arrays ifftshift-ed).  M = 1,
 * FP32 mode, Nt = 2^6..2^13; the problem's reltol/abstol apply (the
 * reference fixes reltol = 1e-5).  At each saveat position (sorted, first 0,
 * last L, as for fl_forward) out_spectra receives the lab-frame spectrum
 * (Nt complex, position-major) and out_pump the pump power -- the reference's
 * "uω_z" and "Ppz" (:222-236), from Tsit5's dense interpolant; stats counts
 * the attempts. */
#define FL_GAIN_CONSTANT 0
#define FL_GAIN_YDFA 1
typedef struct {
    int kind;                 /* FL_GAIN_CONSTANT or FL_GAIN_YDFA */
    double g_const;           /* constant model: gain per metre */
    double gamma_p, sigma_ap, sigma_ep, h_nu_p;  /* pump overlap, cross sections [m^2], h nu_p [J] */
    double gamma_s, area, rho, tau21;            /* signal overlap, core area [m^2], ions [m^-3], [s] */
    double psd_scale;         /* (Nt dt)^2 x repetition rate: |u_w|^2 -> W/Hz */
    double df;                /* bin width [Hz] */
    const double *sigma_as, *sigma_es, *h_nu_s; /* Nt each, FFT bin order (host memory) */
} fl_gain;
int fl_forward_gain(fl_problem *prob, const fl_gain *gain, double pump_power, const double *u0,
                    const double *saveat, int nsave, double *out_spectra, double *out_pump,
                    fl_stats *stats);

/* Forward solve 0 -> L.  Replaces solve_disp_mmf (simulate_disp_mmf.jl:183-207)
 * as used by propagate (propagation.jl:89-123): out_spectra receives the
 * lab-frame spectra cis(D z) ũ(z) at each saveat position (Nt*M*nsave
 * complex, position-major; saveat sorted, first 0, last L, as
 * propagation.jl:60-70 requires).  The forward state is kept (z-checkpoints)
 * for a following fl_adjoint. */
int fl_forward(fl_problem *prob, const double *u0, const double *saveat, int nsave,
               double *out_spectra, fl_stats *stats);

/* Adjoint solve L -> 0 from a lab-frame terminal seed λ(L), using the
 * checkpoints of the last fl_forward on this problem (recomputing the
 * forward field segment by segment).  Replaces solve_adjoint_disp_mmf
 * (sensitivity_disp_mmf.jl:309-332): lambda0 receives sol(0).
 * Fails with FL_NONSYMMETRIC for a gamma tensor that is not
 * permutation-symmetric (sensitivity_disp_mmf.jl:103-112, 239-240). */
int fl_adjoint(fl_problem *prob, const double *lambdaL, double *lambda0, fl_stats *stats);

/* Batched forward + Raman-band objective + adjoint + spectral-phase gradient:
 * the physical-gradient closure of spectral_shaper_model
 * (physics_models.jl:1033-1046) with the band cost/seed of
 * _field_spectral_band_cost (physics_helpers.jl:222-232, dB form :320-326),
 * for nbatch independent launches u0 * cis(phases[:, b]).
 *   u0      (Nt, M) launch spectrum
 *   phases  (Nt, nbatch) vector phase per problem (shared across modes)
 *   mask    Nt bytes, 1 in the band
 *   J       nbatch objective values; grad (Nt, nbatch) ∂J/∂φ summed over
 *           modes (physics_models.jl:732-737); stats nbatch (nullable). */
int fl_phase_gradient_batch(fl_problem *prob, const double *u0, int nbatch,
                            const double *phases, const unsigned char *mask, int log_cost,
                            double *J, double *grad, fl_stats *stats);

/* Same as fl_phase_gradient_batch with one phase per (time bin, mode): the
 * matrix-phase control of _phase_matrix (physics_models.jl:685-704) whose
 * gradient keeps the mode axis.
 *   phases  (Nt, M, nbatch); grad (Nt, M, nbatch) ∂J/∂φ[t, m].
 * For M = 1 this is fl_phase_gradient_batch. */
int fl_mode_phase_gradient_batch(fl_problem *prob, const double *u0, int nbatch,
                                 const double *phases, const unsigned char *mask, int log_cost,
                                 double *J, double *grad, fl_stats *stats);

/* The accepted step positions of the last fl_forward of this problem: the
 * reference's sol.t (the ODESolution's time points with dense output,
 * simulate_disp_mmf.jl:190; used as sol.t by its callers), i.e. 0, the end
 * of every accepted step, and L -- *n_out = naccept + 1 values, of which the
 * first min(cap, *n_out) are written to t_out (cap 0 only queries the
 * count).  FL_EINVAL without a completed preceding fl_forward. */
int fl_forward_times(fl_problem *prob, double *t_out, long cap, long *n_out);

/* Evidence of the last fl_forward (which must have had nsave save
 * positions): FP64 reductions of each saved lab-frame spectrum u on the
 * device, the sums behind propagate's metrics and verify
 * (src/fiberlab/propagation.jl:176-237).  ev_out receives nsave rows of
 * 6 + M values:
 *   [0] Σ_t P(t), P(t) = Σ_m |fft(u_m)(t)|² (the temporal power; times Δt:
 *       the energy in pJ)
 *   [1] max_t P(t) (the peak power in W)
 *   [2] P summed over the first and last max(1, floor(0.05 Nt)) samples
 *       ([2]/[0]: the temporal edge fraction)
 *   [3] Σ_ω S(ω), S = Σ_m |u_m(ω)|² (the spectral power)
 *   [4] S summed over the same edges of fftshift(S) ([4]/[3]: the spectral
 *       edge fraction)
 *   [5] Σ |u|² / |selfsteep| (times Δt/ω0: the photon number, with
 *       selfsteep = fftshift(ωs/ω0) as given to fl_problem_create)
 *   [6 + m] Σ_t |fft(u_m)(t)|² (times Δt: mode m's energy in pJ)
 * FL_EINVAL without such a forward. */
int fl_forward_evidence(fl_problem *prob, int nsave, double *ev_out);

/* One evaluation of the forward right-hand side disp_mmf!
 * (simulate_disp_mmf.jl:25-60) or, with adjoint = 1, of adjoint_disp_mmf!
 * (sensitivity_disp_mmf.jl:32-79) with the forward field u_fwd given
 * directly instead of through the interpolant.  u_in, u_fwd, du_out are
 * (Nt, M) complex host arrays in the interaction picture at position z. */
int fl_rhs_eval(fl_problem *prob, int adjoint, double z, const double *u_in,
                const double *u_fwd, double *du_out);

/* Same with every array already in device memory (HBM-resident timing). */
int fl_phase_gradient_batch_device(fl_problem *prob, const double *d_u0, int nbatch,
                                   const double *d_phases, const unsigned char *d_mask,
                                   int log_cost, double *d_J, double *d_grad,
                                   fl_stats *stats);

/* Device-pointer form of fl_mode_phase_gradient_batch. */
int fl_mode_phase_gradient_batch_device(fl_problem *prob, const double *d_u0, int nbatch,
                                        const double *d_phases, const unsigned char *d_mask,
                                        int log_cost, double *d_J, double *d_grad,
                                        fl_stats *stats);

/* Forward solve that allocates no device memory.  No counterpart in the
 * reference: it serves callers that cannot call cudaMalloc -- host runtimes
 * whose device memory is owned by their own pool allocator, and request loops
 * that must not take cudaMalloc's implicit device synchronisation.  It runs
 * the single-mode FP32 forward stepper on device buffers the caller owns:
 *   d_D, d_selfsteep Nt doubles; d_hR Nt interleaved complex (the
 *   fl_problem_create tables, M = 1); d_u0 Nt complex launch spectrum;
 *   d_saveat nsave positions (sorted, first 0, last L); d_out_spectra
 *   receives Nt*nsave complex lab-frame spectra; stream 0 = default stream.
 * Everything else lives in one file-scope device array of 2 MiB that each GPU
 * loading the library holds until the process exits.  Limit: Nt <= 2^13
 * (larger grids return FL_EUNSUPPORTED); being forward-only it keeps no step
 * log, so the number of steps is bounded only by the attempted-step limit
 * (100000, FL_MAXITERS).  The first call on a device resolves the array's
 * device address (cudaGetSymbolAddress); make that first call before any
 * stream capture.  Every call reuses the same array, so calls that overlap
 * on the GPU (other streams, other host threads) race; the state the solve
 * needs is re-initialised by each call.  The calling thread's current device
 * is restored before the call returns.  An error already pending on the
 * thread is reported as FL_ECUDA and left pending.  Invalid save positions
 * or a non-finite or zero launch return FL_EINVAL. */
int fl_forward_noalloc(int device, int nt, const double *d_D, double gamma, const double *d_hR,
                       const double *d_selfsteep, double one_m_fR, double L, double reltol,
                       double abstol, const double *d_u0, const double *d_saveat, int nsave,
                       double *d_out_spectra, void *stream, fl_stats *stats);

/* ------------------------------------------------------------------------
 * Serving: continuous batching of independent solves.  No counterpart in the
 * reference (which solves one problem per call); it serves the request
 * streams of the reference's callers (propagate / the adjoint model's
 * physical gradient, physics_models.jl:1033-1046) without changing the
 * per-solve arithmetic: each request runs the same stepper as fl_forward /
 * fl_phase_gradient_batch, alone in its slot.
 *
 * A server owns a progress thread.  Requests are grouped by shape (Nt, M,
 * precision) into buckets of slots; each chunk of slots is advanced by a
 * bounded number of right-hand-side evaluations per launch on its own
 * stream, and between launches finished slots are retired (results copied
 * to the caller's buffers) and queued requests admitted into free slots, in
 * arrival order (within an optional cap on requests in flight).
 * New chunks are allocated while the HBM budget allows.  All server calls
 * are thread-safe.  Problems referenced by requests must outlive them.
 * ------------------------------------------------------------------------ */
#define FL_REQ_FORWARD 0        /* output: lab-frame field at L */
#define FL_REQ_BAND_GRADIENT 1  /* outputs: Raman-band J and ∂J/∂φ */

typedef struct {
    size_t hbm_budget_bytes;  /* slot workspaces (default 120 GB) */
    int evals_per_launch;     /* RHS evaluations per slot per launch (default 48) */
    int checkpoints;          /* per-slot z-checkpoints (power of 2, default 256) */
    int segment_steps;        /* recompute sub-segment length (default 128); a band-gradient
                                 request of more than checkpoints x segment_steps accepted
                                 forward steps recomputes more instead of failing; the step
                                 log holds one entry per allowed attempted step (400000) */
    int max_active_ctas;      /* cap on requests in flight, counted in CTAs per transform (one
                                 per single-CTA slot, M x cluster CTAs per multimode slot);
                                 0: no cap beyond slots and the HBM budget */
} fl_server_opts;

typedef struct {
    fl_problem *prob;         /* tables, grid, tolerances */
    int kind;                 /* FL_REQ_FORWARD or FL_REQ_BAND_GRADIENT */
    double L;                 /* fiber length of this request; <= 0: the problem's */
    const double *u0;         /* (Nt, M) complex launch spectrum, copied at submit */
    const double *phase;      /* band gradient: Nt launch phase (shared by modes), copied */
    const unsigned char *mask;/* band gradient: Nt band mask, copied */
    int log_cost;
    double *out_field;        /* forward: (Nt, M) complex lab field at L, written on completion */
    double *out_grad;         /* band gradient: Nt, written on completion */
} fl_request;

typedef struct {
    long submitted, completed, in_flight, queued;
    int slots, chunks;
    size_t hbm_bytes;         /* workspace bytes allocated */
    long launches;
} fl_server_info;

int fl_server_create(fl_ctx *ctx, const fl_server_opts *opts, fl_server **out);
int fl_server_destroy(fl_server *srv);
/* Queue one request; returns its id.  FL_OOM_ADMISSION when one slot of its
 * shape exceeds the HBM budget, FL_EUNSUPPORTED for shapes not built. */
int fl_server_submit(fl_server *srv, const fl_request *req, long *id);
/* FL_EBUSY while running; otherwise the request's final status (its
 * outputs are written) with its stats, J and submit-to-completion latency. */
int fl_server_poll(fl_server *srv, long id, fl_stats *stats, double *J, double *latency_ms);
/* Block until done or timeout_ms elapses (FL_TIMEOUT). */
int fl_server_wait(fl_server *srv, long id, double timeout_ms, fl_stats *stats, double *J,
                   double *latency_ms);
int fl_server_info_get(fl_server *srv, fl_server_info *info);

#ifdef __cplusplus
}
#endif
#endif
