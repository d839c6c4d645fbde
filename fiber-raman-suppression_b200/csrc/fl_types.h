// fl_types.h -- slot descriptors and solver state shared by the host runtime
// and the single-mode solver kernel.  Plain C layout (no CUDA types).
#pragma once
#include <stdint.h>

namespace fl {

enum SlotMode : int {
    MODE_FORWARD = 0,        // forward only (propagate)
    MODE_BAND_GRADIENT = 1,  // forward + Raman-band objective + adjoint + phase gradient
    MODE_SEEDED_ADJOINT = 2  // forward + adjoint from a caller-supplied terminal seed
};

// Terminal objective of MODE_BAND_GRADIENT (its cost and adjoint seed);
// the values of FL_OBJ_* in the C-ABI header.
enum SlotObjective : int {
    OBJ_RAMAN_BAND = 0,   // mode-summed band fraction
    OBJ_FUNDAMENTAL = 1,  // band fraction of mode 1
    OBJ_WORST_MODE = 2,   // log-sum-exp of the per-mode band fractions
    OBJ_RAMAN_PEAK = 3    // strongest in-band bin (summed over modes) over the total
};

enum SlotPhase : int {
    PH_FWD_INIT = 0,
    PH_FWD = 1,
    PH_SEED = 2,
    PH_REC = 3,
    PH_ADJ_INIT = 4,
    PH_ADJ = 5,
    PH_FINAL = 6,
    PH_DONE = 7,
    PH_EVAL_FWD = 8,  // multimode: one forward RHS evaluation (unit parity)
    PH_EVAL_ADJ = 9   // multimode: one adjoint RHS evaluation
};

// status codes (same values as the public FL_* codes)
enum : int {
    ST_OK = 0,
    ST_NONFINITE = 2,
    ST_DT_UNDERFLOW = 3,
    ST_MAXITERS = 4,
    ST_CAPACITY = 9,
    ST_CHECK = 14            // checked build: a state index left its buffer's bounds
};

// Per-slot pointers and parameters.  The forward solve and its recompute
// run in precision RF (float in the default mode, double in the FP64 mode),
// the adjoint in RA (double): typed buffers are void pointers whose element
// type is stated beside them.  Field-sized buffers hold N values.
struct SlotDesc {
    // tables (shared by all slots of one fiber/grid); [0] float, [1] double
    const double* Dturns;   // D/(2 pi), turns per metre
    const void* Heff[2];    // cx: hR * (-1)^k  (fftshift folded in)
    const void* ss[2];      // real: selfsteep = fftshift(ωs/ω0)
    const void* tw[2];      // cx: exp(-2 pi i k / N), k < N
    double gamma, one_m_fR;
    double L, reltol, abstol;
    int mode, log_cost;
    int objective;          // SlotObjective of MODE_BAND_GRADIENT
    double obj_tau;         // worst-mode smoothness τ
    int nsave;
    int ck_cap;             // checkpoint slots K (power of two)
    int seg_cap;            // steps per recompute segment buffer
    int step_cap;           // step-log capacity
    long max_iters;         // attempted-step limit per integration
    // caller data
    const double* zsave;    // nsave save positions (sorted, first 0, last L)
    double* save_out;       // nsave * N complex doubles, lab frame
    const double* u0;       // N complex doubles: launch spectrum (shaped)
    const unsigned char* mask;  // N band mask
    const double* lamL;     // N complex doubles: caller terminal seed (lab frame)
    double* lam0_out;       // N complex doubles (nullable)
    double* grad_out;       // N doubles (nullable)
    double* uL_out;         // N complex doubles: lab field at L (nullable)
    // workspace
    double* u[2];           // FP64 forward states
    double* lam[2];         // FP64 adjoint states
    void* kf[7];            // forward stages, cx<RF>
    void* ka[7];            // adjoint stages, cx<RA>
    void* scr[2];           // per-thread scratch fields, cx<double>-sized
    double* esv;            // error partial, N complex doubles
    double* skv;            // error weights, N doubles
    double* ck_u;           // ck_cap * N complex doubles
    void* ck_k1;            // ck_cap * N cx<RF>
    double* steplog;        // 2 * step_cap doubles (z_n, dt_n)
    void* seg;              // seg_cap * 5 * N cx<RF>: dense interpolant
};

struct SlotState {
    int phase, status;
    int cur, kperm;          // forward: u buffer index, FSAL permutation
    int acur, akperm;        // adjoint: same
    int nsteps, ck_stride, seg, save_idx;
    int rec_pos;             // replayed steps within the current segment
    int stage;               // stage of the attempt in progress (0 = none)
    int sub;                 // sub-segment (seg_cap steps) of the segment being replayed
    double cz, cdt;          // z and signed dt of the attempt in progress
    double aprop;            // adjoint: controller proposal before a segment clip
    double z, dt, qold;      // forward integrator
    double az, adt, aqold;   // adjoint integrator
    double abstol_adj;
    double J;
    long naccept, nreject, nf;
    long a_naccept, a_nreject, a_nf;
    long iters, a_iters;
    long nrec;               // forward steps recomputed for the adjoint
    int dense;               // the forward kept every step's interpolant: no recompute
};

// ---------------------------------------------------------------------------
// Padded row lengths of the multimode contraction tables: the pair axis
// (M(M+1)/2) padded to 4 and the mode axis padded to 2 (vector loads).
__host__ __device__ constexpr int mm_gp(int M) { return (M * (M + 1) / 2 + 3) & ~3; }
__host__ __device__ constexpr int mm_mp(int M) { return (M + 1) & ~1; }
// The adjoint of an FP32-forward batch with M >= 6 modes on whole 128-point
// tiles runs mixed: λ and everything linear in it in FP64, while the forward
// field's transform and pair products (known to FP32 accuracy) run in FP32
// and the contractions on the tensor cores (3xTF32).
// the largest K (rank padded to 8) of the low-rank form: half the pair depth
__host__ __device__ constexpr int mm_krmax(int M) {
    return ((((M * (M + 1) / 2 + 7) & ~7) / 2) + 7) & ~7;
}
__host__ __device__ constexpr bool mm_adj_mixed(int M, int N, int fp64) {
    return !fp64 && M >= 6 && N % 128 == 0;
}

// ---------------------------------------------------------------------------
// Multimode (M > 1) slots.  One right-hand-side evaluation runs as a chain of
// kernels over every active slot (mode transforms, pair convolutions, per-time
// contractions), and a control kernel advances each slot's integrator between
// evaluations.  Fields are mode-major: element (t, m) of an (Nt, M) field sits
// at t + Nt*m, as in the reference's column-major arrays.
struct MmDesc {
    // tables shared by all slots of one problem; [0] float, [1] double
    const double* Dturns;   // M*N: D/(2 pi), turns per metre
    const void* Heff[2];    // cx: hR * (-1)^k
    const void* ss[2];      // real: fftshift(ωs/ω0)
    const void* tw[2];      // cx: exp(-2 pi i k / N)
    const void* G[2];       // M*M*GP: G[(i*M + j)*GP + q] (pair q = (k <= l); GP = NP padded to 4)
    const double* Ga;       // NP*M*MP: the same values as Ga[(j*NP + q)*MP + i] (MP = M padded to 2)
    const float* Gtc;       // M >= 6: the tensor-core B operand (G split hi/lo, shared-memory image)
    const float* Gtcs;      // M >= 6: the symmetric B operand (rows: pairs i <= j, split hi/lo)
    // low-rank form of the pair contraction (rank > 0; FP32 batches, M >= 6):
    // Σ_q G[ij][q] X_q = Σ_k U[ij][k] Z_k with Z_k = Σ_q V[q][k] X_q, k < rank
    int rank;
    const float* Vz;        // B of the Z GEMM: rows k (rank padded to 16), K = pairs, V[q][k]
    const float* Utc;       // B of the forward contraction: rows ij, K = k (rank padded to 8)
    const float* Utcs;      // B of the adjoint's D': rows p = (i <= j), K = k
    int M, NP, N, fp64;     // modes, pairs M(M+1)/2, points, forward precision
    int adj_mixed;          // mm_adj_mixed(M, N, fp64): mixed-precision adjoint
    int nparts;             // error partial sums per evaluation (M x CTAs per transform)
    double one_m_fR;
    double L, reltol, abstol;
    int mode, log_cost, nsave;
    int objective;          // SlotObjective of MODE_BAND_GRADIENT
    double obj_tau;         // worst-mode smoothness τ
    int phase_per_mode;     // gradient: 1 = one phase per (t, m); 0 = phase shared by the modes
    int ck_cap, seg_cap, step_cap;
    long max_iters;
    // caller data
    const double* zsave;
    double* save_out;       // nsave * M*N complex doubles, lab frame
    const double* u0;       // M*N complex doubles
    const unsigned char* mask;  // N band mask
    const double* lamL;     // M*N complex doubles
    double* lam0_out;       // M*N complex doubles (nullable)
    double* grad_out;       // N or M*N doubles (nullable)
    double* uL_out;         // M*N complex doubles (nullable)
    // integrator workspace
    double* u[2];           // FP64 forward states
    double* lam[2];         // FP64 adjoint states
    void* kf[7];            // forward stages, cx<RF>
    void* ka[7];            // adjoint stages, cx<double>
    void* probe;            // initial-step probe derivative, cx<double>-sized
    double* esv;            // error partial, M*N complex doubles
    double* skv;            // error weights, M*N doubles
    double* part;           // error partial sums (nparts doubles)
    double* ck_u;           // ck_cap * M*N complex doubles
    void* ck_k1;            // ck_cap * M*N cx<RF>
    double* steplog;        // 2 * step_cap doubles
    void* seg;              // seg_cap * 5 * M*N cx<RF>
    // right-hand-side workspace (cx<double>-sized so both precisions fit)
    void* ut;               // M*N: forward field in time
    void* lt;               // M*N: adjoint field in time
    void* sq;               // NP*N real: pair sequences S (forward) / S' (adjoint)
    void* cq;               // NP*N real: adjoint Im X, then its Raman correlation
    void* eta;              // M*N: nonlinear term in time
};

struct MmState {
    int phase, status;
    int cur, kperm, acur, akperm;
    int nsteps, ck_stride, seg, save_idx, rec_pos, stage;
    int sub;                // sub-segment (seg_cap steps) of the segment being replayed
    double cz, cdt, aprop;
    double z, dt, qold;
    double az, adt, aqold;
    double abstol_adj, J;
    double ez, ezload;      // position of the pending evaluation and of the forward field it reads
    double dprobe;          // initial step: d1 of the launch
    long naccept, nreject, nf;
    long a_naccept, a_nreject, a_nf;
    long iters, a_iters;
    long nrec;              // forward steps recomputed for the adjoint
    int dense;              // the forward kept every step's interpolant: no recompute
    int ck_pend;            // checkpoint slot + 1 the next step's first prologue stores (0: none)
};

// ---------------------------------------------------------------------------
// Pump-gain single-mode forward solve (disp_gain_smf!, forward only): the
// stepper's slot descriptor (tables, launch u0, state u[2], stages kf[7],
// scratch scr[2], error buffers esv/skv) plus the gain model.  The state is
// [P_pump; ũ]; g(ω) multiplies ũ/2 and dP/dz = g_P P.
struct GainDesc {
    SlotDesc s;
    int kind;               // 0 constant gain, 1 Yb-doped fiber rate equations
    double g_const;         // constant model: g per metre on every bin (g_P = -1)
    double r12c, r21c;      // rate equations: R12 = r12c P, R21 = r21c P
    double inv_tau;         // 1 / τ21
    double gpe, gpa;        // g_P = gpe n2 - gpa n1
    const double* wa;       // W12 = Σ_b wa[b] |u_b|², W21 = Σ_b we[b] |u_b|² (FFT bin order)
    const double* we;
    const double* sA;       // g_b = sE[b] n2 - sA[b] n1
    const double* sE;
    double pump0;           // P_pump at z = 0 [W]
    double* pump_save;      // s.nsave pump powers at s.zsave (s.save_out holds the spectra)
};
struct GainOut {
    long naccept, nreject, nf;
    int status;
    double z_end, pump_L;
};

}  // namespace fl
