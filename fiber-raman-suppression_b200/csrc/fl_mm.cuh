// fl_mm.cuh -- multimode (M > 1) GMMNLSE stepper.
//
// One right-hand-side evaluation of every active slot runs as a chain of
// kernels; a control kernel then consumes the derivative and advances each
// slot's Tsit5 integrator (accept/reject, checkpoints, dense output, the
// checkpoint replay and the adjoint) to its next evaluation.  Kernels skip
// slots whose pending evaluation is not theirs (forward vs adjoint, FP32 vs
// FP64), so one round serves a mixed batch.
//
// Forward RHS (src/simulation/simulate_disp_mmf.jl:25-60), for each slot:
//   prologue  (mode m)  stage input, e^{iD_m z}, F            -> u_t[m]
//   pairs     (q = k<=l, two per task)  P_q = Re(u_k u_l*);
//             S_q = (1-fR) P_q + N⁻¹ F⁻¹(Heff F P_q)          -> S[q]
//   contract  (time t)  η_i = Σ_j (Σ_q G[i,j,q] S_q) u_j        -> η[i]
//   epilogue  (mode m)  dũ_m = i e^{-iD_m z} τ F⁻¹(η_m)/N
// with G[i,j,q] = γ[i,j,k,l] + γ[i,j,l,k] (k < l), γ[i,j,k,k] (k = l): the
// reference's δK = Σ_kl γ_ijkl Re(u_k u_l*) and its Raman convolution δR,
// both linear in the symmetric pair products, contracted once.
//
// Adjoint RHS (src/simulation/sensitivity_disp_mmf.jl:32-79, helpers
// :93-215), for a permutation-symmetric γ (the gate at :103-112):
//   prologue  λ_t = F(e^{iDz} τ λ̃), u_t = F(e^{iDz} ũ(z))
//   imx       (time t)  Im X_ij = Σ_kl γ_klij Im(λ_k u_l*)
//   pairs     (two P's or two Im X's per task)
//             S'_q = 2(1-fR) P_q + h∗P_q,   C_q = h̃⋆ImX_q = N⁻¹F⁻¹(conj(Heff) F ImX_q)
//   contract  (time t)  η_j = Σ_i λ_i δKR1_ij - (1-fR) Σ_i λ_i* δ2_ij
//                              + 2i Σ_i C_ij u_i
//             δKR1_ij = Σ_q G S'_q,  δ2_ij = Σ_q G u_k u_l
//   epilogue  dλ̃ = i e^{-iDz} F⁻¹(η)/N
// The reference's two Raman terms (calc_λ_∂fR2c∂uc!, calc_λc_∂fR∂uc!) are
// complex conjugates of one another (both reduce to the correlation h̃⋆ of
// X = Σ γ λ_t u_t* with the time-reversed, half-period-shifted response), so
// their sum is 2i·h̃⋆(Im X); the conjugate Kerr term reduces to
// -(1-fR) F⁻¹(Σ λ_t* δ2) because F⁻¹(conj(λω)) = conj(λ_t)/N.
//
// Precision: as in the single-mode stepper, the forward evaluations run in
// RF (FP32 by default) with FP64 phase arguments, state, error norm and
// reductions; the adjoint runs in FP64.
#pragma once
#include "fl_cfft.cuh"
#include "fl_sm.cuh"
#include "fl_types.h"

namespace fl {

__host__ __device__ __forceinline__ bool mm_adjoint_phase(int ph) {
    return ph == PH_ADJ_INIT || ph == PH_ADJ || ph == PH_EVAL_ADJ;
}
__host__ __device__ __forceinline__ bool mm_rhs_phase(int ph) {
    return ph == PH_FWD_INIT || ph == PH_FWD || ph == PH_REC || ph == PH_ADJ_INIT ||
           ph == PH_ADJ || ph == PH_EVAL_FWD || ph == PH_EVAL_ADJ;
}
// the pending evaluation of this slot runs in precision R
template <typename R>
__device__ __forceinline__ bool mm_takes(const MmDesc& d, const MmState& st) {
    if (!mm_rhs_phase(st.phase)) return false;
    const bool fp64 = mm_adjoint_phase(st.phase) || d.fp64;
    return (sizeof(R) == 8) == fp64;
}

// pair q (k <= l, row-major over k) -> (k, l)
__host__ __device__ __forceinline__ void pair_kl(int q, int M, int& k, int& l) {
    k = 0;
    int rowlen = M;
    while (q >= rowlen) {
        q -= rowlen;
        k++;
        rowlen--;
    }
    l = k + q;
}

// physical buffer of logical stage i under the FSAL permutation
__device__ __forceinline__ void* mm_kp(void* const* k, int perm, int i) {
    const int p = (perm && (i == 0 || i == 6)) ? 6 - i : i;
    return k[p];
}

// complex load/store of a field element in precision R
template <typename R>
__device__ __forceinline__ cx<double> ldc(const void* p, size_t i) {
    return up(static_cast<const cx<R>*>(p)[i]);
}
// runtime precision (fp64 = stored as cx<double>)
__device__ __forceinline__ cx<double> ldcr(const void* p, size_t i, bool fp64) {
    return fp64 ? static_cast<const cx<double>*>(p)[i] : up(static_cast<const cx<float>*>(p)[i]);
}
__device__ __forceinline__ void stcr(void* p, size_t i, cx<double> v, bool fp64) {
    if (fp64) static_cast<cx<double>*>(p)[i] = v;
    else static_cast<cx<float>*>(p)[i] = down<float>(v);
}

// One transform group: a CTA (C = 1) or a cluster of C CTAs (see
// fl_cfft.cuh).  g is the thread's index in the group, TT the group's thread
// count; a thread owns the positions g + TT*s.
template <typename R, int LOGN, int LOGE, int C>
struct MmGroup {
    using CS = ClusterShape<LOGN, LOGE, C>;
    static constexpr int N = CS::N, E = CS::E, TT = CS::TT, T = CS::T;
    // per-CTA exchange buffer bytes
    static constexpr size_t XBYTES =
        C == 1 ? SmemPlan<R, LOGN>::BYTES : cluster_xbytes<R, LOGN, C>();
    static constexpr size_t SMEM =
        XBYTES + sizeof(cx<R>) * Twiddles<R, LOGN>::SIZE + 32 * sizeof(double);
    int rank, g;
    unsigned char* sm;
    double* red;
    Twiddles<R, LOGN> tw;

    __device__ __forceinline__ void sync() const {
        if constexpr (C == 1) __syncthreads();
        else cluster_sync_all();
    }
    // every CTA of the group calls it (uniform early exits only before it)
    __device__ __forceinline__ void init(const MmDesc& d, unsigned char* smraw) {
        rank = C == 1 ? 0 : (int)(blockIdx.x % C);
        g = rank * T + threadIdx.x;
        sm = smraw;
        cx<R>* tws = reinterpret_cast<cx<R>*>(smraw + XBYTES);
        red = reinterpret_cast<double*>(tws + Twiddles<R, LOGN>::SIZE);
        Twiddles<R, LOGN>::fill(tws, static_cast<const cx<R>*>(d.tw[sizeof(R) == 8]));
        sync();
        tw = Twiddles<R, LOGN>::at(tws);
    }
    __device__ __forceinline__ void fft(cx<R> (&v)[E]) const {
        if constexpr (C == 1) block_fft<R, LOGN, LOGE>(v, sm, tw);
        else cluster_fft<R, LOGN, LOGE, C>(v, reinterpret_cast<cx<R>*>(sm), tw, g);
    }
};

// ---------------------------------------------------------------------------
// prologue: stage input of mode m and its transform(s) to time
// ---------------------------------------------------------------------------
template <typename R, int LOGN, int LOGE, int CL>
__global__ void __launch_bounds__(MmGroup<R, LOGN, LOGE, CL>::T, 1)
    mm_prologue_kernel(const MmDesc* __restrict__ descs, const MmState* __restrict__ states,
                       const int* __restrict__ active) {
    using G = MmGroup<R, LOGN, LOGE, CL>;
    constexpr int N = G::N, E = G::E, T = G::T, TT = G::TT;
    constexpr int P = sizeof(R) == 8;
    using C = cx<R>;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int slot = active[blockIdx.y];
    const MmDesc& d = descs[slot];
    const int m = blockIdx.x / CL;
    if (m >= d.M) return;
    const MmState st = states[slot];
    // a mixed-precision adjoint (mm_adj_mixed) transforms λ in the FP64
    // kernel and the forward field in the FP32 one
    const bool fwd_field = sizeof(R) == 4 && d.adj_mixed && mm_rhs_phase(st.phase) &&
                           mm_adjoint_phase(st.phase);
    if (!mm_takes<R>(d, st) && !fwd_field) return;
    G grp;
    grp.init(d, smraw);
    const int tid = grp.g;  // index in the transform group
    const size_t NM = (size_t)N * d.M, off = (size_t)m * N;
    const int ph = st.phase;
    const bool adj = mm_adjoint_phase(ph);
    const double* Dt = d.Dturns + off;
    C v[E];

    if (!fwd_field) {
        // ---- stage input (FP64 accumulation, as the single-mode stepper)
        if (ph == PH_EVAL_FWD || ph == PH_EVAL_ADJ) {
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = down<R>(ld2(d.u0, off + tid + TT * s));
        } else if (ph == PH_FWD_INIT || ph == PH_ADJ_INIT) {
            const bool fw = ph == PH_FWD_INIT;
            const double* x0 = fw ? d.u0 : d.lam[0];
            const C* k1 = static_cast<const C*>(fw ? d.kf[0] : d.ka[0]);
            const double sg = fw ? st.cdt : -st.cdt;
#pragma unroll
            for (int s = 0; s < E; s++) {
                const size_t b = off + tid + TT * s;
                const cx<double> x = ld2(x0, b);
                if (st.stage == 0) {
                    v[s] = down<R>(x);
                } else {
                    const C f0 = k1[b];
                    v[s] = mk((R)(x.re + sg * (double)f0.re), (R)(x.im + sg * (double)f0.im));
                }
            }
        } else {
            const bool fw = !adj;
            void* const* K = fw ? d.kf : d.ka;
            const int perm = fw ? st.kperm : st.akperm;
            const int cur = fw ? st.cur : st.acur;
            const double* x = fw ? d.u[cur] : d.lam[cur];
            const double dt = st.cdt;
            if (st.stage < 6) {
                // a checkpoint due at this step's start (set by the control kernel)
                const int ckp = ph == PH_FWD && st.stage == 1 ? st.ck_pend : 0;
                // stage-outer, point-inner over chunks of SC points: each
                // stage's loads of a chunk are in flight together (the
                // per-point sum still runs over the stages in order)
                constexpr int SC = E < 8 ? E : 8;
#pragma unroll
                for (int s0 = 0; s0 < E; s0 += SC) {
                    double ar[SC], ai[SC];
#pragma unroll
                    for (int c = 0; c < SC; c++) ar[c] = ai[c] = 0.0;
#pragma unroll 1
                    for (int j = 0; j < st.stage; j++) {
                        const C* __restrict__ kj = static_cast<const C*>(mm_kp(K, perm, j));
                        const double a = kT5a[st.stage][j];
                        C xk[SC];
#pragma unroll
                        for (int c = 0; c < SC; c++) xk[c] = kj[off + tid + TT * (s0 + c)];
#pragma unroll
                        for (int c = 0; c < SC; c++) {
                            ar[c] += a * (double)xk[c].re;
                            ai[c] += a * (double)xk[c].im;
                        }
                        if (ckp && j == 0) {
#pragma unroll
                            for (int c = 0; c < SC; c++)
                                static_cast<C*>(d.ck_k1)[(size_t)(ckp - 1) * NM + off + tid + TT * (s0 + c)] = xk[c];
                        }
                    }
#pragma unroll
                    for (int c = 0; c < SC; c++) {
                        const size_t b = off + tid + TT * (s0 + c);
                        const cx<double> un = ld2(x, b);
                        if (ckp) st2(d.ck_u, (size_t)(ckp - 1) * NM + b, un);
                        v[s0 + c] = mk((R)(un.re + dt * ar[c]), (R)(un.im + dt * ai[c]));
                    }
                }
            } else {
                double* xnew = fw ? d.u[cur ^ 1] : d.lam[cur ^ 1];
                const bool want_err = ph != PH_REC;
                const double at = fw ? d.abstol : st.abstol_adj, rt = d.reltol;
                // chunks of SC6 points, the six stages' loads of a chunk in
                // flight together (two sums per point: solution and error)
                constexpr int SC6 = E < 4 ? E : 4;
#pragma unroll
                for (int s0 = 0; s0 < E; s0 += SC6) {
                    double ar[SC6], ai[SC6], er[SC6], ei[SC6];
#pragma unroll
                    for (int c = 0; c < SC6; c++) ar[c] = ai[c] = er[c] = ei[c] = 0.0;
#pragma unroll
                    for (int j = 0; j < 6; j++) {
                        const C* __restrict__ kj = static_cast<const C*>(mm_kp(K, perm, j));
                        const double a = kT5a[6][j], bt = kT5bt[j];
                        C xk[SC6];
#pragma unroll
                        for (int c = 0; c < SC6; c++) xk[c] = kj[off + tid + TT * (s0 + c)];
#pragma unroll
                        for (int c = 0; c < SC6; c++) {
                            ar[c] += a * (double)xk[c].re;
                            ai[c] += a * (double)xk[c].im;
                            er[c] += bt * (double)xk[c].re;
                            ei[c] += bt * (double)xk[c].im;
                        }
                    }
#pragma unroll
                    for (int c = 0; c < SC6; c++) {
                        const size_t b = off + tid + TT * (s0 + c);
                        const cx<double> un = ld2(x, b);
                        const cx<double> u1 = mk(un.re + dt * ar[c], un.im + dt * ai[c]);
                        st2(xnew, b, u1);
                        if (want_err) {
                            st2(d.esv, b, mk(dt * er[c], dt * ei[c]));
                            const double m0 = sqrt(un.re * un.re + un.im * un.im);
                            const double m1 = sqrt(u1.re * u1.re + u1.im * u1.im);
                            d.skv[b] = at + fmax(m0, m1) * rt;
                        }
                        v[s0 + c] = down<R>(u1);
                    }
                }
            }
        }

        // ---- to time: forward u_t = F(e^{iDz} ũ); adjoint λ_t = F(e^{iDz} τ λ̃)
        const R* ss = static_cast<const R*>(d.ss[P]);
        C* out = static_cast<C*>(adj ? d.lt : d.ut);
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int t = tid + TT * s;
            v[s] = cmul(v[s], phasor<R>(Dt[t], st.ez));
            if (adj) v[s] = scale(v[s], ss[t]);
        }
        grp.fft(v);
#pragma unroll
        for (int s = 0; s < E; s++) out[off + tid + TT * s] = v[s];
        if (!adj || d.adj_mixed) return;  // (mixed: the FP32 kernel takes the forward field)
    }

    // ---- adjoint: the forward field at ezload, F(e^{iDz} ũ(z))
    if (ph == PH_EVAL_ADJ) {
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = down<R>(ld2(d.lamL, off + tid + TT * s));
    } else {
        const SubSeg sb = sub_segment(d, st);
        const int seg_lo = sb.lo;
        const double zz = st.ezload;
        const double* lg = d.steplog;
        // last stored step starting at or before zz, by bisection
        int n = seg_lo, hi = sb.hi - 1;
        while (n < hi) {
            const int mid = (n + hi + 1) >> 1;
            if (lg[2 * mid] <= zz) n = mid;
            else hi = mid - 1;
        }
        const double zn = lg[2 * n], dtn = lg[2 * n + 1];
        const double th = (zz - zn) / dtn, t2 = th * th, t3 = t2 * th, t4 = t3 * th;
        const size_t base = (size_t)(n - seg_lo) * 5 * NM;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const size_t b = off + tid + TT * s;
            cx<double> c[5];
#pragma unroll
            for (int q = 0; q < 5; q++) c[q] = ldcr(d.seg, base + q * NM + b, d.fp64);
            const double xr = c[0].re + dtn * (th * c[1].re + t2 * c[2].re + t3 * c[3].re + t4 * c[4].re);
            const double xi = c[0].im + dtn * (th * c[1].im + t2 * c[2].im + t3 * c[3].im + t4 * c[4].im);
            v[s] = mk((R)xr, (R)xi);
        }
    }
    grp.sync();  // the exchange buffer is reused
#pragma unroll
    for (int s = 0; s < E; s++) v[s] = cmul(v[s], phasor<R>(Dt[tid + TT * s], st.ez));
    grp.fft(v);
    C* uo = static_cast<C*>(d.ut);
#pragma unroll
    for (int s = 0; s < E; s++) uo[off + tid + TT * s] = v[s];
}

// ---------------------------------------------------------------------------
// pairs: Raman convolutions of the symmetric pair products.  Two real
// sequences of the same kind share one complex transform pair (the kernels
// Heff and conj(Heff) are Hermitian, so their products with the packed
// spectrum stay separated in the real and imaginary parts).  Tasks
// [0, ceil(NP/2)) take the products P_q, and in the adjoint tasks
// [ceil(NP/2), 2 ceil(NP/2)) the Im X_q: packing P (~|u_t|²) with the much
// smaller Im X would leave Im X with the rounding of P.
// ---------------------------------------------------------------------------
template <typename R, int LOGN, int LOGE, int CL>
__global__ void __launch_bounds__(MmGroup<R, LOGN, LOGE, CL>::T, 1)
    mm_pairs_kernel(const MmDesc* __restrict__ descs, const MmState* __restrict__ states,
                    const int* __restrict__ active) {
    using G = MmGroup<R, LOGN, LOGE, CL>;
    constexpr int N = G::N, E = G::E, T = G::T, TT = G::TT;
    constexpr int P = sizeof(R) == 8;
    using C = cx<R>;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int slot = active[blockIdx.y];
    const MmDesc& d = descs[slot];
    const MmState st = states[slot];
    const bool adj = mm_rhs_phase(st.phase) && mm_adjoint_phase(st.phase);
    // a mixed-precision adjoint (mm_adj_mixed) forms the products P of the
    // forward field in the FP32 kernel and the Im X correlations in FP64
    const bool mixed = adj && d.adj_mixed;
    if (!mm_takes<R>(d, st) && !(mixed && sizeof(R) == 4)) return;
    const int M = d.M, NP = d.NP, ntp = (NP + 1) / 2;
    const int unit = blockIdx.x / CL;
    const bool ytask = unit >= ntp;  // correlation of Im X (adjoint only)
    if (ytask && !adj) return;
    if (mixed && ytask != (sizeof(R) == 8)) return;
    // the low-rank form (rank > 0, FP32 kernels only) convolves pairs of the
    // rank sequences Z_k = Σ_q V[q][k] P_q instead of the NP products
    // (and the adjoint correlates the rank sequences Yz_k = Σ_q V[q][k] Y_q)
    const bool zmode = !ytask && d.rank > 0;
    const int nseq = d.rank > 0 ? d.rank : NP;
    const int q0 = 2 * (ytask ? unit - ntp : unit);
    if (q0 >= nseq) return;
    const int q1 = q0 + 1;
    const bool two = q1 < nseq;
    G grp;
    grp.init(d, smraw);
    const int tid = grp.g;  // index in the transform group
    const C* ut = static_cast<const C*>(d.ut);
    const C* H = static_cast<const C*>(d.Heff[P]);
    R* sq = static_cast<R*>(d.sq);
    R* cq = static_cast<R*>(d.cq);
    const R ofr = (R)d.one_m_fR, invn = R(1) / R(N);
    int k0, l0, k1 = 0, l1 = 0;
    pair_kl(q0, M, k0, l0);
    if (two) pair_kl(q1, M, k1, l1);
    C v[E];
    R p0[E], p1[E];
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int t = tid + TT * s;
        if (ytask) {
            p0[s] = cq[(size_t)q0 * N + t];
            p1[s] = two ? cq[(size_t)q1 * N + t] : R(0);
        } else if (zmode) {
            const R* zq = sq + (size_t)NP * N;  // Z_k rows (upper half of the pair table)
            p0[s] = zq[(size_t)q0 * N + t];
            p1[s] = two ? zq[(size_t)q1 * N + t] : R(0);
        } else {
            const C a = ut[(size_t)k0 * N + t], b = ut[(size_t)l0 * N + t];
            p0[s] = a.re * b.re + a.im * b.im;  // Re(u_k u_l*)
            if (two) {
                const C a1 = ut[(size_t)k1 * N + t], b1 = ut[(size_t)l1 * N + t];
                p1[s] = a1.re * b1.re + a1.im * b1.im;
            } else {
                p1[s] = R(0);
            }
        }
        v[s] = mk(p0[s], p1[s]);
    }
    grp.fft(v);
#pragma unroll
    for (int s = 0; s < E; s++) {
        const C h = H[tid + TT * s];
        v[s] = ytask ? cmulc(v[s], h) : cmul(v[s], h);  // conj(Heff): correlation
    }
    conj_all(v);
    grp.fft(v);
    conj_all(v);
    // forward S = (1-fR) P + h∗P; adjoint S' = 2(1-fR) P + h∗P and C = h̃⋆Im X
    const R kf = adj ? R(2) * ofr : ofr;
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int t = tid + TT * s;
        if (ytask) {
            cq[(size_t)q0 * N + t] = v[s].re * invn;
            if (two) cq[(size_t)q1 * N + t] = v[s].im * invn;
        } else {
            sq[(size_t)q0 * N + t] = kf * p0[s] + v[s].re * invn;
            if (two) sq[(size_t)q1 * N + t] = kf * p1[s] + v[s].im * invn;
        }
    }
}

// ---------------------------------------------------------------------------
// epilogue: nonlinear term of mode m back to the interaction frame, stored
// as the stage derivative; the stage-7 error partial of the mode
// ---------------------------------------------------------------------------
template <typename R, int LOGN, int LOGE, int CL>
__global__ void __launch_bounds__(MmGroup<R, LOGN, LOGE, CL>::T, 1)
    mm_epilogue_kernel(const MmDesc* __restrict__ descs, const MmState* __restrict__ states,
                       const int* __restrict__ active) {
    using G = MmGroup<R, LOGN, LOGE, CL>;
    constexpr int N = G::N, E = G::E, T = G::T, TT = G::TT;
    constexpr int P = sizeof(R) == 8;
    using C = cx<R>;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int slot = active[blockIdx.y];
    const MmDesc& d = descs[slot];
    const int m = blockIdx.x / CL;
    if (m >= d.M) return;
    const MmState st = states[slot];
    if (!mm_takes<R>(d, st)) return;
    G grp;
    grp.init(d, smraw);
    const int tid = grp.g;  // index in the transform group
    const size_t off = (size_t)m * N;
    const int ph = st.phase;
    const bool adj = mm_adjoint_phase(ph);
    const C* eta = static_cast<const C*>(d.eta);
    C v[E];
#pragma unroll
    for (int s = 0; s < E; s++) v[s] = conjc(eta[off + tid + TT * s]);
    grp.fft(v);
    const double* Dt = d.Dturns + off;
    const R* ss = static_cast<const R*>(d.ss[P]);
    const R invn = R(1) / R(N);
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int t = tid + TT * s;
        const C y = cmulc(conjc(v[s]), phasor<R>(Dt[t], st.ez));  // e^{-iDz} x
        const R sc = adj ? invn : ss[t] * invn;
        v[s] = mk(-y.im * sc, y.re * sc);  // i y (τ) / N
    }
    if (ph == PH_EVAL_FWD || ph == PH_EVAL_ADJ) {
#pragma unroll
        for (int s = 0; s < E; s++) st2(d.lam0_out, off + tid + TT * s, up(v[s]));
        return;
    }
    C* dst;
    if (ph == PH_FWD_INIT) dst = static_cast<C*>(st.stage == 0 ? d.kf[0] : d.probe);
    else if (ph == PH_ADJ_INIT) dst = static_cast<C*>(st.stage == 0 ? d.ka[0] : d.probe);
    else if (adj) dst = static_cast<C*>(mm_kp(d.ka, st.akperm, st.stage));
    else dst = static_cast<C*>(mm_kp(d.kf, st.kperm, st.stage));
#pragma unroll
    for (int s = 0; s < E; s++) dst[off + tid + TT * s] = v[s];
    // dense interpolant of this mode's part of the step: c0 = ũ_n,
    // c_p = Σ_i r_ip k_i (Tsit5's free 4th-order interpolant).  A replayed
    // step keeps it for the steps of the current sub-segment; a forward
    // attempt keeps it at the step's index while the solve fits the buffer
    // (a rejected attempt is overwritten by its retry), so a solve that fits
    // needs no recompute for its adjoint.
    const SubSeg sb = sub_segment(d, st);
    const bool keep_rec = ph == PH_REC && sb.seg_lo + st.rec_pos >= sb.lo;
    const bool keep_fwd = ph == PH_FWD && d.step_cap > 0 && st.nsteps < d.seg_cap;
    if (st.stage == 6 && (keep_rec || keep_fwd)) {
        const size_t NM = (size_t)N * d.M,
                     base = (size_t)(keep_rec ? sb.seg_lo + st.rec_pos - sb.lo : st.nsteps) * 5 * NM;
        C* sg = static_cast<C*>(d.seg);
        const double* un = d.u[st.cur];
        // pairs of points, the six stored stages' loads of a pair in flight
        // together (the per-point sums run over the stages in order)
#pragma unroll
        for (int s0 = 0; s0 < E; s0 += 2) {
            double cr[2][4], ci[2][4];
#pragma unroll
            for (int c = 0; c < 2; c++)
#pragma unroll
                for (int q = 0; q < 4; q++) cr[c][q] = ci[c][q] = 0.0;
#pragma unroll
            for (int i = 0; i < 7; i++) {
                C ki[2];
#pragma unroll
                for (int c = 0; c < 2; c++)
                    ki[c] = i == 6 ? v[s0 + c]
                                   : static_cast<const C*>(mm_kp(d.kf, st.kperm, i))[off + tid + TT * (s0 + c)];
#pragma unroll
                for (int c = 0; c < 2; c++)
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        cr[c][q] += kT5r[i][q] * (double)ki[c].re;
                        ci[c][q] += kT5r[i][q] * (double)ki[c].im;
                    }
            }
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const size_t b = off + tid + TT * (s0 + c);
                sg[base + b] = down<R>(ld2(un, b));
#pragma unroll
                for (int q = 0; q < 4; q++) sg[base + (q + 1) * NM + b] = mk((R)cr[c][q], (R)ci[c][q]);
            }
        }
    }
    if (st.stage == 6 && (ph == PH_FWD || ph == PH_ADJ)) {
        const double dt = st.cdt, bt7 = kT5bt[6];
        double acc = 0.0;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const size_t b = off + tid + TT * s;
            const cx<double> e6 = ld2(d.esv, b);
            const double er = e6.re + dt * bt7 * (double)v[s].re;
            const double ei = e6.im + dt * bt7 * (double)v[s].im;
            const double w = d.skv[b];
            acc += (er * er + ei * ei) / (w * w);
        }
        const double tot = block_sum<T>(acc, grp.red);
        if (threadIdx.x == 0) d.part[m * CL + grp.rank] = tot;
    }
}

// ---------------------------------------------------------------------------
// per-time contractions (one thread per time point; M at compile time)
// ---------------------------------------------------------------------------
constexpr int kMmTB = 128;  // threads per block of the contraction kernels

// Row lengths of the contraction tables: the pair axis of G padded to a
// multiple of 4 (zeros) so rows load as float4 / double2 vectors, and the
// mode axis of the adjoint table padded to even.
template <int M>
struct MmPairs {
    static constexpr int NP = M * (M + 1) / 2;
    static constexpr int GP = (NP + 3) & ~3;
    static constexpr int MP = (M + 1) & ~1;
};

// acc[0..3] += row[q..q+3] * x[q..q+3] for q in [0, GP)
template <int GP>
__device__ __forceinline__ float dot_row(const float* __restrict__ row, const float (&x)[GP]) {
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
    for (int q = 0; q < GP; q += 4) {
        const float4 g = __ldg(reinterpret_cast<const float4*>(row + q));
        a0 += g.x * x[q];
        a1 += g.y * x[q + 1];
        a2 += g.z * x[q + 2];
        a3 += g.w * x[q + 3];
    }
    return (a0 + a1) + (a2 + a3);
}
template <int GP>
__device__ __forceinline__ double dot_row(const double* __restrict__ row, const double (&x)[GP]) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
    for (int q = 0; q < GP; q += 4) {
        const double2 g0 = __ldg(reinterpret_cast<const double2*>(row + q));
        const double2 g1 = __ldg(reinterpret_cast<const double2*>(row + q + 2));
        a0 += g0.x * x[q];
        a1 += g0.y * x[q + 1];
        a2 += g1.x * x[q + 2];
        a3 += g1.y * x[q + 3];
    }
    return (a0 + a1) + (a2 + a3);
}

// forward: η_i = Σ_j (Σ_q G[i,j,q] S_q) u_j, in precision R
template <typename R, int M>
__device__ __forceinline__ void mm_contract_fwd(const MmDesc& d, int t) {
    using PS = MmPairs<M>;
    constexpr int NP = PS::NP, GP = PS::GP;
    const int N = d.N;
    const cx<R>* ut = static_cast<const cx<R>*>(d.ut);
    const R* sq = static_cast<const R*>(d.sq);
    const R* G = static_cast<const R*>(d.G[sizeof(R) == 8]);
    cx<R>* eta = static_cast<cx<R>*>(d.eta);
    cx<R> u[M];
    R Sv[GP];
#pragma unroll
    for (int j = 0; j < M; j++) u[j] = ut[(size_t)j * N + t];
#pragma unroll
    for (int q = 0; q < GP; q++) Sv[q] = q < NP ? sq[(size_t)q * N + t] : R(0);
#pragma unroll 1
    for (int i = 0; i < M; i++) {
        const R* Gi = G + (size_t)i * M * GP;
        R er = R(0), ei = R(0);
#pragma unroll
        for (int j = 0; j < M; j++) {
            const R dij = dot_row<GP>(Gi + j * GP, Sv);
            er += dij * u[j].re;
            ei += dij * u[j].im;
        }
        eta[(size_t)i * N + t] = mk(er, ei);
    }
}

// adjoint, first pass: Im X_p = Σ_q G[i,j,q] Yh_q for the pairs p = (i <= j),
// Yh_q = (Im(λ_k u_l*) + Im(λ_l u_k*))/2 (k < l), Im(λ_k u_k*) (k = l)
template <int M>
__device__ __forceinline__ void mm_imx(const MmDesc& d, int t) {
    using PS = MmPairs<M>;
    constexpr int NP = PS::NP, GP = PS::GP;
    const int N = d.N;
    const cx<double>* lt = static_cast<const cx<double>*>(d.lt);
    const cx<double>* ut = static_cast<const cx<double>*>(d.ut);
    const double* G = static_cast<const double*>(d.G[1]);
    double* cq = static_cast<double*>(d.cq);
    double Y[GP];
    {
        cx<double> la[M], u[M];
#pragma unroll
        for (int j = 0; j < M; j++) {
            la[j] = lt[(size_t)j * N + t];
            u[j] = ut[(size_t)j * N + t];
        }
        int q = 0;
#pragma unroll
        for (int k = 0; k < M; k++) {
#pragma unroll
            for (int l = k; l < M; l++) {
                const double a = la[k].im * u[l].re - la[k].re * u[l].im;  // Im(λ_k u_l*)
                const double b = la[l].im * u[k].re - la[l].re * u[k].im;
                Y[q++] = k == l ? a : 0.5 * (a + b);
            }
        }
#pragma unroll
        for (int r = NP; r < GP; r++) Y[r] = 0.0;
    }
#pragma unroll 1
    for (int p = 0; p < NP; p++) {
        int i, j;
        pair_kl(p, M, i, j);
        cq[(size_t)p * N + t] = dot_row<GP>(G + ((size_t)i * M + j) * GP, Y);
    }
}

// adjoint, second pass (thread per (t, j)):
//   η_j = Σ_q S'_q g_q - (1-fR) Σ_q (u_k u_l) conj(g_q) + 2i Σ_i C_ij u_i,
//   g_q = Σ_i λ_i G[i,j,q], read from the table Ga[(j*NP + q)*MP + i]
// (a thread per time point for all j read the point's fields once but ran
// 15 % slower on a 10-mode launch list: fewer threads, more registers)
template <int M>
__device__ __forceinline__ void mm_contract_adj(const MmDesc& d, int t, int j) {
    using PS = MmPairs<M>;
    constexpr int NP = PS::NP, MP = PS::MP;
    const int N = d.N;
    const cx<double>* lt = static_cast<const cx<double>*>(d.lt);
    const cx<double>* ut = static_cast<const cx<double>*>(d.ut);
    const double* sq = static_cast<const double*>(d.sq);
    const double* cq = static_cast<const double*>(d.cq);
    const double* Ga = d.Ga + (size_t)j * NP * MP;
    cx<double>* eta = static_cast<cx<double>*>(d.eta);
    const double ofr = d.one_m_fR;
    cx<double> la[MP], u[M];
#pragma unroll
    for (int i = 0; i < M; i++) {
        la[i] = lt[(size_t)i * N + t];
        u[i] = ut[(size_t)i * N + t];
    }
#pragma unroll
    for (int i = M; i < MP; i++) la[i] = mk(0.0, 0.0);
    double er = 0.0, ei = 0.0;
    int q = 0;
#pragma unroll
    for (int k = 0; k < M; k++) {
#pragma unroll
        for (int l = k; l < M; l++) {
            double gr = 0.0, gi = 0.0;
#pragma unroll
            for (int i = 0; i < MP; i += 2) {
                const double2 g = __ldg(reinterpret_cast<const double2*>(Ga + (size_t)q * MP + i));
                gr += g.x * la[i].re + g.y * la[i + 1].re;
                gi += g.x * la[i].im + g.y * la[i + 1].im;
            }
            const double s = sq[(size_t)q * N + t];
            const cx<double> w = cmul(u[k], u[l]);
            // S' g - (1-fR) w conj(g)
            er += s * gr - ofr * (w.re * gr + w.im * gi);
            ei += s * gi - ofr * (w.im * gr - w.re * gi);
            q++;
        }
    }
    // 2i Σ_i C_ij u_i, C symmetric stored per pair (min, max)
#pragma unroll
    for (int i = 0; i < M; i++) {
        const int a = i < j ? i : j, b = i < j ? j : i;
        const int p = a * M - a * (a - 1) / 2 + (b - a);
        const double c = cq[(size_t)p * N + t];
        er -= 2.0 * c * u[i].im;
        ei += 2.0 * c * u[i].re;
    }
    eta[(size_t)j * N + t] = mk(er, ei);
}

// which = 0: forward contraction in R; 1: adjoint Im X; 2: adjoint assembly
template <typename R, int M>
__global__ void __launch_bounds__(kMmTB)
    mm_contract_kernel(const MmDesc* __restrict__ descs, const MmState* __restrict__ states,
                       const int* __restrict__ active, int which) {
    const int slot = active[blockIdx.y];
    const MmDesc& d = descs[slot];
    if (d.M != M) return;
    const MmState st = states[slot];
    if (!mm_takes<R>(d, st)) return;
    const bool adj = mm_adjoint_phase(st.phase);
    if (which == 0 && adj) return;
    if (which != 0 && (!adj || sizeof(R) != 8)) return;
    const int g = blockIdx.x * kMmTB + threadIdx.x;
    if (which == 2) {
        if (g >= d.N * M) return;
        mm_contract_adj<M>(d, g % d.N, g / d.N);
        return;
    }
    if (g >= d.N) return;
    if (which == 0) mm_contract_fwd<R, M>(d, g);
    else mm_imx<M>(d, g);
}

// ---------------------------------------------------------------------------
// control: consume the derivative of the last evaluation and advance the
// integrator to its next evaluation (one CTA per slot, block-uniform state)
// ---------------------------------------------------------------------------
constexpr int kMmCtl = 512;
constexpr int kMmMaxModes = 10;  // modes of the built multimode shapes

struct MmCtl {
    const MmDesc& d;
    MmState& st;
    double* red;
    size_t NM;
    int N;

    __device__ double sum(double v) { return block_sum<kMmCtl>(v, red); }
    __device__ double maxv(double v) { return block_max<kMmCtl>(v, red); }

    __device__ void restore_checkpoint(int seg) {
        for (size_t i = threadIdx.x; i < NM; i += kMmCtl) {
            st2(d.u[0], i, ld2(d.ck_u, (size_t)seg * NM + i));
            stcr(d.kf[0], i, ldcr(d.ck_k1, (size_t)seg * NM + i, d.fp64), d.fp64);
        }
        st.cur = 0;
        st.kperm = 0;
        st.rec_pos = 0;
        st.stage = 0;
    }

    __device__ void store_checkpoint(int slotc, const double* un, const void* k1) {
        for (size_t i = threadIdx.x; i < NM; i += kMmCtl) {
            st2(d.ck_u, (size_t)slotc * NM + i, ld2(un, i));
            stcr(d.ck_k1, (size_t)slotc * NM + i, ldcr(k1, i, d.fp64), d.fp64);
        }
    }

    // lab frame e^{+iDz} x of a stored FP64 field into out
    __device__ void lab(const double* x, double z, double* out) {
        for (size_t i = threadIdx.x; i < NM; i += kMmCtl) {
            const cx<double> a = ld2(x, i);
            const cx<double> p = phasor<double>(d.Dturns[i], z);
            st2(out, i, mk(a.re * p.re - a.im * p.im, a.re * p.im + a.im * p.re));
        }
    }

    // --------------------------------------------------------------- consume
    __device__ void consume() {
        const int ph = st.phase;
        const double L = d.L, dtmin = kEps * L;
        if (ph == PH_FWD_INIT || ph == PH_ADJ_INIT) {
            const bool fw = ph == PH_FWD_INIT;
            const double* x0 = fw ? d.u0 : d.lam[0];
            const double at = fw ? d.abstol : st.abstol_adj, rt = d.reltol;
            const void* k1 = fw ? d.kf[0] : d.ka[0];
            const bool k64 = fw ? d.fp64 != 0 : true;
            if (st.stage == 0) {
                double s0 = 0.0, s1 = 0.0;
                for (size_t i = threadIdx.x; i < NM; i += kMmCtl) {
                    const cx<double> x = ld2(x0, i);
                    const double ax = sqrt(x.re * x.re + x.im * x.im);
                    const double sk = at + ax * rt;
                    s0 += (ax / sk) * (ax / sk);
                    const cx<double> f = ldcr(k1, i, k64);
                    const double af = sqrt(f.re * f.re + f.im * f.im);
                    s1 += (af / sk) * (af / sk);
                }
                const double d0 = sqrt(sum(s0) / (double)NM);
                const double d1 = sqrt(sum(s1) / (double)NM);
                const double dt0 = initdt_first(d0, d1, L);
                double r;
                if (!isfinite(d1)) r = -dtmin;
                else if (dt0 < 10 * kEps) r = -fmax(1e-6, dtmin);
                else r = dt0;
                if (r > 0.0) {
                    st.cdt = r;
                    st.dprobe = d1;
                    st.stage = 1;
                    return;
                }
                st.cdt = -r;
            } else {
                double s2 = 0.0, nd = 0.0;
                for (size_t i = threadIdx.x; i < NM; i += kMmCtl) {
                    const cx<double> x = ld2(x0, i);
                    const double sk = at + sqrt(x.re * x.re + x.im * x.im) * rt;
                    const cx<double> f0 = ldcr(k1, i, k64), f1 = ldcr(d.probe, i, k64);
                    const double dr = f1.re - f0.re, di = f1.im - f0.im;
                    s2 += (dr * dr + di * di) / (sk * sk);
                    nd += (dr != 0.0 || di != 0.0) ? 1.0 : 0.0;
                }
                const double d2 = sqrt(sum(s2) / (double)NM) / st.cdt;
                const double ndt = sum(nd);
                st.cdt = initdt_final(st.cdt, st.dprobe, d2, ndt, dtmin, L);
            }
            st.stage = 0;
            if (fw) {
                st.z = 0.0;
                st.dt = st.cdt;
                st.qold = kQoldInit;
                st.cur = 0;
                st.kperm = 0;
                st.nsteps = 0;
                st.ck_stride = 1;
                st.ck_pend = 0;
                st.naccept = st.nreject = st.iters = 0;
                st.nf = 3;
                if (d.ck_cap > 0) store_checkpoint(0, d.u0, d.kf[0]);
                st.save_idx = 0;
                while (st.save_idx < d.nsave && d.zsave[st.save_idx] == 0.0) {
                    double* o = d.save_out + (size_t)st.save_idx * 2 * NM;
                    for (size_t i = threadIdx.x; i < NM; i += kMmCtl) st2(o, i, ld2(d.u0, i));
                    st.save_idx++;
                }
                st.phase = PH_FWD;
            } else {
                st.az = L;
                st.adt = -st.cdt;
                st.aqold = kQoldInit;
                st.a_nf = 3;
                st.acur = 0;
                st.akperm = 0;
                st.phase = PH_ADJ;
            }
            return;
        }
        if (ph == PH_FWD || ph == PH_REC) {
            if (st.stage < 6) {
                if (st.stage == 1) st.ck_pend = 0;  // stored by this round's prologue
                st.stage++;
                return;
            }
            st.stage = 0;
            const double z = st.cz, dt = st.cdt;
            const double* u = d.u[st.cur];
            const bool f64 = d.fp64 != 0;
            if (ph == PH_REC) {
                // (the epilogue has stored this step's dense interpolant)
                st.cur ^= 1;
                st.kperm ^= 1;
                st.rec_pos++;
                st.nrec++;
                const SubSeg sb = sub_segment(d, st);
                if (sb.seg_lo + st.rec_pos >= sb.hi) st.phase = st.a_nf == 0 ? PH_ADJ_INIT : PH_ADJ;
                return;
            }
            double acc = 0.0;
            for (int m = 0; m < d.nparts; m++) acc += d.part[m];
            const double EEst = sqrt(acc / (double)NM);
            if (!isfinite(EEst)) {
                st.status = ST_NONFINITE;
                st.phase = PH_DONE;
                return;
            }
            double q11;
            const double q = pi_q(EEst, st.qold, q11);
            st.nf += 6;
            if (EEst > 1.0) {
                st.nreject++;
                st.dt = dt / fmin(1.0 / kQmin, q11 / kGamma);
                return;
            }
            st.naccept++;
            if (d.step_cap > 0) {  // step_cap 0: forward only, nothing kept for an adjoint
                if (st.nsteps >= d.step_cap) {
                    st.status = ST_CAPACITY;
                    st.phase = PH_DONE;
                    return;
                }
                if (threadIdx.x == 0) {
                    d.steplog[2 * st.nsteps] = z;
                    d.steplog[2 * st.nsteps + 1] = dt;
                }
            }
            double znew = z + dt;
            if (fabs(znew - d.L) < 100.0 * kEps * fmax(z, d.L)) znew = d.L;
            // save positions in (z, znew) and on an interior step end (those
            // at L take the final state)
            while (st.save_idx < d.nsave && d.zsave[st.save_idx] > z &&
                   (d.zsave[st.save_idx] < znew ||
                    (d.zsave[st.save_idx] == znew && znew < d.L))) {
                const double zs = d.zsave[st.save_idx];
                const double th = (zs - z) / dt;
                double bi[7];
                for (int s = 0; s < 7; s++) {
                    double b = 0.0, tp = th;
                    for (int qq = 0; qq < 4; qq++) {
                        b += kT5r[s][qq] * tp;
                        tp *= th;
                    }
                    bi[s] = b;
                }
                double* o = d.save_out + (size_t)st.save_idx * 2 * NM;
                for (size_t i = threadIdx.x; i < NM; i += kMmCtl) {
                    double xr = 0.0, xi = 0.0;
                    for (int s = 0; s < 7; s++) {
                        const cx<double> ks = ldcr(mm_kp(d.kf, st.kperm, s), i, f64);
                        xr += bi[s] * ks.re;
                        xi += bi[s] * ks.im;
                    }
                    const cx<double> un = ld2(u, i);
                    const cx<double> x = mk(un.re + dt * xr, un.im + dt * xi);
                    const cx<double> p = phasor<double>(d.Dturns[i], zs);
                    st2(o, i, mk(x.re * p.re - x.im * p.im, x.re * p.im + x.im * p.re));
                }
                st.save_idx++;
            }
            st.nsteps++;
            st.z = znew;
            st.cur ^= 1;
            st.kperm ^= 1;
            st.qold = fmax(EEst, kQoldInit);
            st.dt = fmin(fmax((q == 1.0) ? dt : dt / q, dtmin), d.L);
            if (d.ck_cap > 0 && (st.nsteps % st.ck_stride) == 0) {
                int slotc = st.nsteps / st.ck_stride;
                if (slotc >= d.ck_cap) {
                    for (int j = 1; j < d.ck_cap / 2; j++) {
                        __syncthreads();
                        for (size_t i = threadIdx.x; i < NM; i += kMmCtl) {
                            st2(d.ck_u, (size_t)j * NM + i, ld2(d.ck_u, (size_t)2 * j * NM + i));
                            stcr(d.ck_k1, (size_t)j * NM + i,
                                 ldcr(d.ck_k1, (size_t)2 * j * NM + i, f64), f64);
                        }
                    }
                    st.ck_stride *= 2;
                    slotc = st.nsteps / st.ck_stride;
                }
                if (znew == d.L) {
                    __syncthreads();
                    store_checkpoint(slotc, d.u[st.cur], mm_kp(d.kf, st.kperm, 0));
                } else {
                    // the next step's stage-1 prologue loads exactly u_n and
                    // k1 in all of its mode groups: it stores the checkpoint
                    // (one CTA copying 2-4 MB here was latency-bound)
                    st.ck_pend = slotc + 1;
                }
            }
            if (st.z == d.L) {
                for (int si = st.save_idx; si < d.nsave; si++)
                    lab(d.u[st.cur], d.L, d.save_out + (size_t)si * 2 * NM);
                if (d.uL_out) lab(d.u[st.cur], d.L, d.uL_out);
                st.save_idx = d.nsave;
                st.phase = d.mode == MODE_FORWARD ? PH_DONE : PH_SEED;
            }
            return;
        }
        if (ph == PH_ADJ) {
            if (st.stage < 6) {
                st.stage++;
                return;
            }
            st.stage = 0;
            const double z = st.cz, dt = st.cdt;
            const double zlo = d.steplog[2 * sub_segment(d, st).lo];
            double acc = 0.0;
            for (int m = 0; m < d.nparts; m++) acc += d.part[m];
            const double EEst = sqrt(acc / (double)NM);
            if (!isfinite(EEst)) {
                st.status = ST_NONFINITE;
                st.phase = PH_DONE;
                return;
            }
            double q11;
            const double q = pi_q(EEst, st.aqold, q11);
            st.a_nf += 6;
            if (EEst > 1.0) {
                st.a_nreject++;
                st.adt = st.adt / fmin(1.0 / kQmin, q11 / kGamma);
                return;
            }
            st.a_naccept++;
            double znew = z + dt;
            if (fabs(znew - zlo) < 100.0 * kEps * fmax(z, zlo)) znew = zlo;
            st.az = znew;
            st.acur ^= 1;
            st.akperm ^= 1;
            st.aqold = fmax(EEst, kQoldInit);
            const double adt = -dt;
            double dtn = fmin(fmax((q == 1.0) ? adt : adt / q, dtmin), d.L);
            if (adt < st.aprop) dtn = fmax(dtn, st.aprop);  // shortened for a segment start
            st.adt = -dtn;
            if (st.az == zlo) {
                if (st.sub > 0) {  // the previous sub-segment of this segment
                    st.sub--;
                    __syncthreads();
                    restore_checkpoint(st.seg);
                    st.phase = PH_REC;
                } else if (st.seg == 0) {
                    st.phase = PH_FINAL;
                } else {
                    st.seg--;
                    st.sub = last_sub(d, st, st.seg);
                    __syncthreads();
                    restore_checkpoint(st.seg);
                    st.phase = PH_REC;
                }
            }
        }
    }

    // --------------------------------------------------------------- advance
    __device__ void advance() {
        const double L = d.L, dtmin = kEps * L;
        for (;;) {
            const int ph = st.phase;
            if (ph == PH_DONE || ph == PH_EVAL_FWD || ph == PH_EVAL_ADJ) return;
            if (ph == PH_SEED) {
                __syncthreads();
                seed();
                continue;
            }
            if (ph == PH_FINAL) {
                const double* lam = d.lam[st.acur];
                for (size_t i = threadIdx.x; i < NM; i += kMmCtl) {
                    const cx<double> l = ld2(lam, i);
                    if (d.lam0_out) st2(d.lam0_out, i, l);
                    if (d.grad_out && d.phase_per_mode) {
                        const cx<double> us = ld2(d.u0, i);
                        d.grad_out[i] = 2.0 * (l.im * us.re - l.re * us.im);
                    }
                }
                if (d.grad_out && !d.phase_per_mode) {
                    // phase shared by the modes: ∂J/∂φ summed over modes
                    for (int t = threadIdx.x; t < N; t += kMmCtl) {
                        double g = 0.0;
                        for (int m = 0; m < d.M; m++) {
                            const size_t i = (size_t)m * N + t;
                            const cx<double> l = ld2(lam, i), us = ld2(d.u0, i);
                            g += 2.0 * (l.im * us.re - l.re * us.im);
                        }
                        d.grad_out[t] = g;
                    }
                }
                st.phase = PH_DONE;
                continue;
            }
            if (ph == PH_FWD_INIT) {
                if (st.stage == 0)
                    for (size_t i = threadIdx.x; i < NM; i += kMmCtl) st2(d.u[0], i, ld2(d.u0, i));
                st.ez = st.stage == 0 ? 0.0 : st.cdt;
                return;
            }
            if (ph == PH_FWD || ph == PH_REC) {
                if (st.stage == 0) {
                    if (ph == PH_REC) {
                        const int n = st.seg * st.ck_stride + st.rec_pos;
                        st.cz = d.steplog[2 * n];
                        st.cdt = d.steplog[2 * n + 1];
                    } else {
                        if (++st.iters > d.max_iters) {
                            st.status = ST_MAXITERS;
                            st.phase = PH_DONE;
                            continue;
                        }
                        double adt = fmax(fmin(fabs(st.dt), L), dtmin);
                        const double rem = L - st.z;
                        if (adt > rem) adt = rem;
                        if (adt <= dtmin && rem > dtmin) {
                            st.status = ST_DT_UNDERFLOW;
                            st.phase = PH_DONE;
                            continue;
                        }
                        st.cz = st.z;
                        st.cdt = adt;
                    }
                    st.stage = 1;
                }
                st.ez = st.cz + kT5c[st.stage] * st.cdt;
                return;
            }
            if (ph == PH_ADJ_INIT) {
                st.ez = st.stage == 0 ? L : L - st.cdt;
                st.ezload = st.stage == 0 ? L : fmax(st.ez, d.steplog[2 * sub_segment(d, st).lo]);
                return;
            }
            // PH_ADJ
            if (st.stage == 0) {
                if (++st.a_iters > d.max_iters) {
                    st.status = ST_MAXITERS;
                    st.phase = PH_DONE;
                    continue;
                }
                // segment starts are made transparent to the controller (no
                // sliver step before one; the pre-clip proposal is restored)
                const double zlo = d.steplog[2 * sub_segment(d, st).lo];
                const double prop = fmax(fmin(fabs(st.adt), L), dtmin);
                const double rem = st.az - zlo;
                double adt = prop;
                if (adt >= rem) adt = rem;
                else if (adt > 0.5 * rem) adt = 0.5 * rem;
                st.aprop = prop;
                st.cz = st.az;
                st.cdt = -adt;
                st.stage = 1;
            }
            st.ez = st.ezload = st.cz + kT5c[st.stage] * st.cdt;
            return;
        }
    }

    // terminal seed λ̃(L) into lam[0], then the replay of the last segment
    __device__ void seed() {
        const double* uf = d.u[st.cur];
        double* lam = d.lam[0];
        if (d.mode == MODE_BAND_GRADIENT) {
            // The objectives of physics_helpers.jl:222-302.  Each seed is
            // u(L) times a real factor per (mode, bin) -- a_m (sel - r_m) --
            // so the interaction-frame seed is ũ(L) times the same factor:
            //   band         a = 1/E,          r = J, sel = band mask
            //   fundamental  a_0 = 1/E_0, 0 on the other modes, r = J
            //   worst mode   a_m = w_m/E_m (w = softmax τ r over the modes
            //                with energy), r_m = mode m's band fraction
            //   peak         a = 1/E, r = J, sel = the strongest in-band bin
            //                (mode-summed energy, lowest index among equals)
            const int M = d.M, obj = d.objective;
            double a[kMmMaxModes], r[kMmMaxModes];
            double cost;
            int pk = -1;
            if (obj == OBJ_FUNDAMENTAL || obj == OBJ_WORST_MODE) {
                double tm[kMmMaxModes];
                for (int m = 0; m < M; m++) {
                    double et = 0.0, eb = 0.0;
                    for (int t = threadIdx.x; t < N; t += kMmCtl) {
                        const double e = energy(ld2(uf, (size_t)m * N + t));
                        et += e;
                        if (d.mask[t]) eb += e;
                    }
                    tm[m] = sum(et);
                    const double bm = sum(eb);
                    r[m] = tm[m] > 0.0 ? bm / tm[m] : 0.0;
                    a[m] = 0.0;
                }
                if (obj == OBJ_FUNDAMENTAL) {
                    cost = r[0];
                    a[0] = 1.0 / tm[0];
                    for (int m = 1; m < M; m++) r[m] = 0.0;
                } else {
                    double rmax = -1.0;
                    int K = 0;
                    for (int m = 0; m < M; m++)
                        if (tm[m] > 0.0) {
                            rmax = fmax(rmax, r[m]);
                            K++;
                        }
                    double den = 0.0;
                    for (int m = 0; m < M; m++)
                        if (tm[m] > 0.0) den += exp(d.obj_tau * (r[m] - rmax));
                    cost = rmax + (log(den) - log((double)K)) / d.obj_tau;
                    for (int m = 0; m < M; m++)
                        a[m] = tm[m] > 0.0 ? exp(d.obj_tau * (r[m] - rmax)) / den / tm[m] : 0.0;
                }
            } else {
                double et = 0.0, eb = 0.0, emax = -1.0;
                for (int t = threadIdx.x; t < N; t += kMmCtl) {
                    double e = 0.0;
                    for (int m = 0; m < M; m++) e += energy(ld2(uf, (size_t)m * N + t));
                    et += e;
                    if (d.mask[t]) {
                        eb += e;
                        emax = fmax(emax, e);
                    }
                }
                const double tot = sum(et);
                double band = sum(eb);
                if (obj == OBJ_RAMAN_PEAK) {
                    band = maxv(emax);
                    // lowest index as the largest key N - t (maxv folds from 0)
                    double key = 0.0;
                    for (int t = threadIdx.x; t < N; t += kMmCtl) {
                        double e = 0.0;
                        for (int m = 0; m < M; m++) e += energy(ld2(uf, (size_t)m * N + t));
                        if (d.mask[t] && e == band) key = fmax(key, (double)(N - t));
                    }
                    pk = N - (int)maxv(key);
                }
                cost = band / tot;
                for (int m = 0; m < M; m++) {
                    a[m] = 1.0 / tot;
                    r[m] = cost;
                }
            }
            double sc = 1.0;
            st.J = cost;
            if (d.log_cost) {  // physics_helpers.jl:320-326
                st.J = 10.0 * log10(fmax(cost, 1e-15));
                sc = cost <= 1e-15 ? 0.0 : 10.0 / (log(10.0) * cost);
            }
            for (size_t i = threadIdx.x; i < NM; i += kMmCtl) {
                const int m = (int)(i / N), t = (int)(i % N);
                const cx<double> x = ld2(uf, i);
                const double sel = obj == OBJ_RAMAN_PEAK ? (t == pk ? 1.0 : 0.0)
                                                         : (d.mask[t] ? 1.0 : 0.0);
                const double f = a[m] * (sel - r[m]) * sc;
                st2(lam, i, mk(x.re * f, x.im * f));
            }
        } else {
            st.J = 0.0;
            for (size_t i = threadIdx.x; i < NM; i += kMmCtl) {
                const cx<double> x = ld2(d.lamL, i);
                const cx<double> p = phasor<double>(d.Dturns[i], d.L);
                st2(lam, i, mk(x.re * p.re + x.im * p.im, x.im * p.re - x.re * p.im));
            }
        }
        __syncthreads();
        double mx = 0.0;
        bool finite = true;
        for (size_t i = threadIdx.x; i < NM; i += kMmCtl) {
            const cx<double> x = ld2(lam, i);
            const double a = sqrt(x.re * x.re + x.im * x.im);
            if (!isfinite(a)) finite = false;
            mx = fmax(mx, a);
        }
        const double scl = maxv(finite ? mx : INFINITY);
        if (!isfinite(scl)) {
            st.status = ST_NONFINITE;
            st.phase = PH_DONE;
            return;
        }
        st.abstol_adj = scl == 0.0 ? d.abstol : d.abstol * scl;  // sensitivity_disp_mmf.jl:324-325
        st.nrec = 0;
        st.acur = 0;
        st.akperm = 0;
        st.a_naccept = st.a_nreject = st.a_nf = st.a_iters = 0;
        // every step's interpolant is in the buffer when the forward fit it:
        // the adjoint runs L -> 0 without recompute or stops
        st.dense = st.nsteps <= d.seg_cap ? 1 : 0;
        if (st.dense) {
            st.seg = 0;
            st.sub = 0;
            st.phase = PH_ADJ_INIT;
            return;
        }
        st.seg = (st.nsteps + st.ck_stride - 1) / st.ck_stride - 1;
        st.sub = last_sub(d, st, st.seg);
        restore_checkpoint(st.seg);
        st.phase = PH_REC;
    }
};

}  // namespace fl
