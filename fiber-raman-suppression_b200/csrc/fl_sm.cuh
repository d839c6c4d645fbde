// fl_sm.cuh -- single-mode GMMNLSE stepper: one CTA owns one problem (slot)
// and runs its whole adaptive Tsit5 solve, the checkpoint-replay recompute
// and the adjoint solve as a state machine whose state lives in global
// memory, so a launch can advance a slot by a bounded number of attempted
// steps (serving) or run it to completion (plain drop-in).
//
// Reference path: forward RHS src/simulation/simulate_disp_mmf.jl:25-60,
// adjoint RHS src/simulation/sensitivity_disp_mmf.jl:32-79 (with the helper
// terms :93-215), drivers simulate_disp_mmf.jl:183-207 and
// sensitivity_disp_mmf.jl:309-332, band objective
// src/fiberlab/physics_helpers.jl:222-232, phase gradient
// src/fiberlab/physics_models.jl:1042.
//
// For M = 1 the RHS is evaluated in an algebraically identical form with
// fewer transforms (4 forward, 5 adjoint instead of 4 and 14):
//   forward  dũ = i e^{-iDz} τ F⁻¹[((1-fR) I + h∗I) u_t],  I = γ|u_t|²
//   adjoint  dλ̃ = i e^{-iDz} F⁻¹[ λ_t (2(1-fR) I + h∗I) - (1-fR) γ λ_t* u_t²
//                                 + 2i (h̃⋆Y) u_t ],  Y = γ Im(λ_t u_t*)
// where u_t = F(e^{iDz} ũ), λ_t = F(e^{iDz} τ λ̃), h∗ is the Raman convolution
// with the fftshift folded into Heff = hR (-1)^k, and h̃⋆ the correlation
// (conj(Heff)).  The two Raman terms of the reference adjoint (:93-132) are
// complex conjugates of each other and combine into the single real
// correlation of Y; h∗I and h̃⋆Y share one complex transform pair.
//
// Precision: the forward solve and its recompute run in RF (FP32 in the
// default mode) with FP64 phase arguments, FP64 state accumulation and an FP64
// error norm; the dense interpolant is stored in RF.  The adjoint integration
// (the gradient accumulation along z) runs in RA = FP64: an FP32 adjoint
// amplifies its round-off through the modulation-instability gain of the
// anomalous-dispersion fiber and misses 1e-3 gradient accuracy (measured
// 2e-3..7e-3 on the Nt = 2^13 band-objective problem; 4e-6 in FP64).
#pragma once
#include "fl_fft.cuh"
#include "fl_types.h"

namespace fl {

// Tsitouras (2011) 5(4) pair, as used by OrdinaryDiffEq's Tsit5.
static __device__ __constant__ double kT5c[7] = {0.0, 0.161, 0.327, 0.9, 0.9800255409045097, 1.0, 1.0};
static __device__ __constant__ double kT5a[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {0.161, 0, 0, 0, 0, 0},
    {-0.008480655492356989, 0.335480655492357, 0, 0, 0, 0},
    {2.897153057105493, -6.359448489975075, 4.3622954328695815, 0, 0, 0},
    {5.325864828439257, -11.748883564062828, 7.4955393428898365, -0.09249506636175525, 0, 0},
    {5.86145544294642, -12.92096931784711, 8.159367898576159, -0.071584973281401,
     -0.028269050394068383, 0},
    {0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081,
     2.324710524099774}};
static __device__ __constant__ double kT5bt[7] = {-0.00178001105222577714, -0.0008164344596567469,
                                           0.007880878010261995,    -0.1447110071732629,
                                           0.5823571654525552,      -0.45808210592918697,
                                           0.015151515151515152};
// free 4th-order interpolant b_i(θ) = Σ_p r[i][p] θ^(p+1)
static __device__ __constant__ double kT5r[7][4] = {
    {1.0, -2.763706197274826, 2.9132554618219126, -1.0530884977290216},
    {0.0, 0.13169999999999998, -0.2234, 0.1017},
    {0.0, 3.9302962368947516, -5.941033872131505, 2.490627285651253},
    {0.0, -12.411077166933676, 30.33818863028232, -16.548102889244902},
    {0.0, 37.50931341651104, -88.1789048947664, 47.37952196281928},
    {0.0, -27.896526289197286, 65.09189467479366, -34.87065786149661},
    {0.0, 1.5, -4.0, 2.5}};

// PI controller defaults of OrdinaryDiffEq for a 5th-order method
constexpr double kBeta1 = 7.0 / 50.0, kBeta2 = 2.0 / 25.0, kGamma = 0.9;
constexpr double kQmin = 0.2, kQmax = 10.0, kQoldInit = 1e-4;
constexpr double kEps = 2.220446049250313e-16;

// exp(+i D z) from the FP64 phase in turns reduced to [-1/2, 1/2] before the
// sincos of the working precision.
template <typename R>
__device__ __forceinline__ cx<R> phasor(double dturn, double z);
template <>
__device__ __forceinline__ cx<float> phasor<float>(double dturn, double z) {
    double ph = dturn * z;
    ph -= rint(ph);
    float s, c;
    sincospif(2.0f * (float)ph, &s, &c);
    return mk(c, s);
}
template <>
__device__ __forceinline__ cx<double> phasor<double>(double dturn, double z) {
    double ph = dturn * z;
    ph -= rint(ph);
    double s, c;
    sincospi(2.0 * ph, &s, &c);
    return mk(c, s);
}

__device__ __forceinline__ cx<double> ld2(const double* p, int b) {
    const double2 v = reinterpret_cast<const double2*>(p)[b];
    return mk(v.x, v.y);
}
__device__ __forceinline__ void st2(double* p, int b, cx<double> v) {
    reinterpret_cast<double2*>(p)[b] = make_double2(v.re, v.im);
}
// |x|² rounded the same way wherever it is evaluated (no contraction choice
// left to the compiler), so energies of one field compare exactly
__device__ __forceinline__ double energy(cx<double> x) {
    return __fma_rn(x.re, x.re, __dmul_rn(x.im, x.im));
}
template <typename R>
__device__ __forceinline__ cx<double> up(cx<R> a) {
    return mk((double)a.re, (double)a.im);
}
template <typename R>
__device__ __forceinline__ cx<R> down(cx<double> a) {
    return mk((R)a.re, (R)a.im);
}

// deterministic block reductions (fixed shuffle tree, fixed warp order)
template <int T>
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < T / 32; w++) s += red[w];
    return s;
}
template <int T>
__device__ __forceinline__ double block_max(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < T / 32; w++) s = fmax(s, red[w]);
    return s;
}

// Shared-memory layout of the stepper: [transform buffer][32 reduction
// doubles][FP32 twiddles][FP64 twiddles].  red points at the reduction area.
template <typename R, int LOGN>
__device__ __forceinline__ const cx<R>* smem_twiddles(double* red) {
    unsigned char* p = reinterpret_cast<unsigned char*>(red) + 32 * sizeof(double);
    if constexpr (sizeof(R) == 8)
        p += sizeof(cx<float>) * Twiddles<float, LOGN>::SIZE;
    return reinterpret_cast<const cx<R>*>(p);
}

// Copy both precisions' twiddle tables into shared memory (the FP64 table is
// absent when no adjoint will run) and wait for the block.
template <int LOGN>
__device__ __forceinline__ void load_twiddles(const SlotDesc& d, double* red) {
    Twiddles<float, LOGN>::fill(const_cast<cx<float>*>(smem_twiddles<float, LOGN>(red)),
                                (const cx<float>*)d.tw[0]);
    if (d.tw[1])
        Twiddles<double, LOGN>::fill(const_cast<cx<double>*>(smem_twiddles<double, LOGN>(red)),
                                     (const cx<double>*)d.tw[1]);
    __syncthreads();
}

// The field handed between the state machine and the out-of-line RHS, as
// element s = bin t + T s of thread t: in the transform buffer in shared
// memory where that buffer holds a complex FP64 field (Nt <= 2^13), else in
// a per-thread array in local memory.  Each thread only touches its own
// bins, so handing over needs no barrier; the RHS synchronises once after
// reading its input, before its first transform exchange overwrites the
// buffer.
template <typename C, int LOGN, int LOGE>
struct FieldIO {
    static constexpr bool SMEM = !SmemPlan<double, LOGN>::SPLIT;
    static constexpr int T = FftShape<LOGN, LOGE>::T;
    C* p;
    __device__ __forceinline__ C& operator[](int s) const {
        if constexpr (SMEM) return p[pad(threadIdx.x + T * s)];
        else return p[s];
    }
};

// ---------------------------------------------------------------------------
// Tensor memory as the right-hand side's per-thread scratch (sm_100a).
//
// Each RHS evaluation parks two fields between its transforms -- u_t in the
// forward, λ_t and u_t in the adjoint -- and every thread only ever reads
// back the bins it wrote.  At Nt = 2^12..2^13 those fields fit the SM's
// 256 KB of tensor memory, which this kernel's FFT leaves unused: the CTA
// allocates it once (tcgen05.alloc) and threads move their own values with
// tcgen05.st / tcgen05.ld (32x32b shape: a warp addresses the 32 lanes of
// its lane quarter, warp % 4, and each thread its own lane's columns), in
// place of two per-slot fields in global memory (five 128 KB round trips
// per FP64 adjoint evaluation).  Layout: lane 32 (w % 4) + (t % 32), columns
// (w / 4) * 8E + f * 4E + [0, 4E) for field f of warp w: room for two FP64
// fields, which also holds the FP32 forward's one.
constexpr uint32_t kNoTmem = 0xFFFFFFFFu;

template <int LOGN, int LOGE>
struct TmLayout {
    using S = FftShape<LOGN, LOGE>;
    static constexpr int E = S::E, T = S::T;
    static constexpr int WARPS = T / 32;
    static constexpr int PER_Q = (WARPS + 3) / 4;      // warps sharing a lane quarter
    static constexpr int COLS_WARP = 8 * E;            // two FP64 fields (4 words per value)
    static constexpr int NEED = COLS_WARP * PER_Q;
    // allocation: a power of two >= 32 columns
    static constexpr int COLS = NEED <= 32 ? 32 : NEED <= 64 ? 64 : NEED <= 128 ? 128
                              : NEED <= 256 ? 256 : 512;
    // only for the grids whose CTAs are few per SM (their allocations then
    // never wait on one another): 2^12 (2 CTAs, 256 columns each) and 2^13
    static constexpr bool ENABLED = (LOGN == 12 || LOGN == 13) && NEED <= 512 && T >= 256;
};

__device__ __forceinline__ void tm_st16(uint32_t a, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16};" ::"r"(a),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
        "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
        "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void tm_ld16(uint32_t a, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(a)
        : "memory");
}
__device__ __forceinline__ void tm_wait_st() {
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tm_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void pack_words(cx<float> v, uint32_t* w) {
    w[0] = __float_as_uint(v.re);
    w[1] = __float_as_uint(v.im);
}
__device__ __forceinline__ void pack_words(cx<double> v, uint32_t* w) {
    w[0] = (uint32_t)__double2loint(v.re);
    w[1] = (uint32_t)__double2hiint(v.re);
    w[2] = (uint32_t)__double2loint(v.im);
    w[3] = (uint32_t)__double2hiint(v.im);
}
__device__ __forceinline__ void unpack_words(const uint32_t* w, cx<float>& v) {
    v.re = __uint_as_float(w[0]);
    v.im = __uint_as_float(w[1]);
}
__device__ __forceinline__ void unpack_words(const uint32_t* w, cx<double>& v) {
    v.re = __hiloint2double((int)w[1], (int)w[0]);
    v.im = __hiloint2double((int)w[3], (int)w[2]);
}

// This thread's two scratch fields (its own E bins) in precision R.
template <typename R, int LOGN, int LOGE>
struct TmScratch {
    using L = TmLayout<LOGN, LOGE>;
    static constexpr int E = L::E;
    static constexpr int WPV = (int)(2 * sizeof(R) / 4);  // words per complex value
    static constexpr int VPC = 16 / WPV;                  // values per 16-word chunk
    static constexpr int CH = E / VPC;                    // chunks per field
    static_assert(!L::ENABLED || E % VPC == 0, "a field is whole chunks");
    uint32_t a0;  // this warp's field 0, column 0
    __device__ explicit TmScratch(uint32_t tm) {
        const int w = threadIdx.x >> 5;
        a0 = tm + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)((w >> 2) * L::COLS_WARP);
    }
    __device__ __forceinline__ uint32_t addr(int f, int c) const {
        return a0 + (uint32_t)(f * 4 * E + c * 16);
    }
    __device__ __forceinline__ void put(int f, const cx<R> (&v)[E]) const {
#pragma unroll
        for (int c = 0; c < CH; c++) {
            uint32_t w[16];
#pragma unroll
            for (int j = 0; j < VPC; j++) pack_words(v[c * VPC + j], w + j * WPV);
            tm_st16(addr(f, c), w);
        }
        tm_wait_st();
    }
    __device__ __forceinline__ void get(int f, int c, cx<R> (&o)[VPC]) const {
        uint32_t w[16];
        tm_ld16(addr(f, c), w);
        tm_wait_ld();
#pragma unroll
        for (int j = 0; j < VPC; j++) unpack_words(w + j * WPV, o[j]);
    }
    __device__ __forceinline__ void get2(int c, cx<R> (&o0)[VPC], cx<R> (&o1)[VPC]) const {
        uint32_t w0[16], w1[16];
        tm_ld16(addr(0, c), w0);
        tm_ld16(addr(1, c), w1);
        tm_wait_ld();
#pragma unroll
        for (int j = 0; j < VPC; j++) {
            unpack_words(w0 + j * WPV, o0[j]);
            unpack_words(w1 + j * WPV, o1[j]);
        }
    }
};

// Allocate the CTA's scratch columns (warp 0) and publish the address through
// the shared-memory slot; every thread of the CTA calls it.  The caller frees
// them with tm_free before the CTA exits.
template <int LOGN, int LOGE>
__device__ __forceinline__ uint32_t tm_alloc(uint32_t* slot) {
    using L = TmLayout<LOGN, LOGE>;
    if constexpr (!L::ENABLED) {
        return kNoTmem;
    } else {
        if ((threadIdx.x >> 5) == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             (uint32_t)__cvta_generic_to_shared(slot)),
                         "r"(L::COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        return *slot;
    }
}
template <int LOGN, int LOGE>
__device__ __forceinline__ void tm_free(uint32_t tm) {
    using L = TmLayout<LOGN, LOGE>;
    if constexpr (L::ENABLED) {
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if ((threadIdx.x >> 5) == 0)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm),
                         "r"(L::COLS));
    }
}

// Block-level pieces of one problem's solve in RHS precision R.
template <typename R, int LOGN, int LOGE>
struct SmSolver {
    using S = FftShape<LOGN, LOGE>;
    static constexpr int N = S::N, E = S::E, T = S::T;
    static constexpr int P = sizeof(R) == 8 ? 1 : 0;  // table precision index
    using C = cx<R>;
    using IO = FieldIO<C, LOGN, LOGE>;

    const SlotDesc& d;
    void* sm;       // padded transform buffer
    double* red;    // 32 doubles
    Twiddles<R, LOGN> tw;  // two-level table in shared memory
    const C* __restrict__ Heff;
    const R* __restrict__ ss;
    const double* __restrict__ Dturns;
    C* scr0;
    C* scr1;
    uint32_t tm;  // tensor-memory scratch of the CTA, or kNoTmem: scr0 / scr1 in global memory
    using TMS = TmScratch<R, LOGN, LOGE>;
    static constexpr int VPC = TMS::VPC;

    __device__ SmSolver(const SlotDesc& dd, void* smem, double* r, uint32_t tmaddr = kNoTmem)
        : d(dd), sm(smem), red(r), tw(Twiddles<R, LOGN>::at(smem_twiddles<R, LOGN>(r))),
          Heff((const C*)dd.Heff[P]), ss((const R*)dd.ss[P]), Dturns(dd.Dturns),
          scr0((C*)dd.scr[0]), scr1((C*)dd.scr[1]), tm(tmaddr) {}

    __device__ __forceinline__ static int bin(int s) { return threadIdx.x + T * s; }

    // One right-hand-side evaluation, forward (adj = false) or adjoint, as a
    // runtime loop over its transforms so the kernel holds one copy of the
    // FFT code (inverse transforms run as conj∘F∘conj):
    //   forward  f0: ũ e^{iDz} -F-> u_t       f1: (γ|u_t|², 0) -F->
    //            f2: ·Heff -F⁻¹-> N h∗I       f3: ((1-fR)I + h∗I) u_t -F⁻¹->
    //            post: dũ = i e^{-iDz} τ (·)/N
    //   adjoint  f0: λ̃ e^{iDz} τ -F-> λ_t     f1: ũ(z) e^{iDz} -F-> u_t
    //            f2: (I, Y) -F-> X            f3: split X into Î, Ŷ;
    //                Heff Î + i conj(Heff) Ŷ -F⁻¹-> N (h∗I + i h̃⋆Y)
    //            f4: η -F⁻¹->                post: dλ̃ = i e^{-iDz} (·)/N
    // load_u(v) fills v with the forward field ũ(z) for the adjoint.
    template <class LoadU>
    __device__ void rhs(const bool adj, const double z, C (&v)[E], LoadU&& load_u) {
        const R g = (R)d.gamma, ofr = (R)d.one_m_fR, invn = R(1) / R(N);
        const int nfft = adj ? 5 : 4;
#pragma unroll 1
        for (int f = 0; f < nfft; f++) {
            bool inv = false;
            const int op = adj ? 8 + f : f;
            if (op == 0) {
#pragma unroll
                for (int s = 0; s < E; s++) v[s] = cmul(v[s], phasor<R>(Dturns[bin(s)], z));
            } else if (op == 1) {
                if (TmLayout<LOGN, LOGE>::ENABLED && tm != kNoTmem) {
                    TMS(tm).put(0, v);
#pragma unroll
                    for (int s = 0; s < E; s++) v[s] = mk(g * abs2(v[s]), R(0));
                } else {
#pragma unroll
                    for (int s = 0; s < E; s++) {
                        scr0[bin(s)] = v[s];
                        v[s] = mk(g * abs2(v[s]), R(0));
                    }
                }
            } else if (op == 2) {
#pragma unroll
                for (int s = 0; s < E; s++) v[s] = cmul(v[s], Heff[bin(s)]);
                inv = true;
            } else if (op == 3) {
                if (TmLayout<LOGN, LOGE>::ENABLED && tm != kNoTmem) {
                    const TMS ts(tm);
#pragma unroll
                    for (int c = 0; c < TMS::CH; c++) {
                        C u[VPC];
                        ts.get(0, c, u);
#pragma unroll
                        for (int j = 0; j < VPC; j++) {
                            const int s = c * VPC + j;
                            const R fac = ofr * (g * abs2(u[j])) + v[s].re * invn;
                            v[s] = scale(u[j], fac);
                        }
                    }
                } else {
#pragma unroll
                    for (int s = 0; s < E; s++) {
                        const C ut = scr0[bin(s)];
                        const R fac = ofr * (g * abs2(ut)) + v[s].re * invn;
                        v[s] = scale(ut, fac);
                    }
                }
                inv = true;
            } else if (op == 8) {
#pragma unroll
                for (int s = 0; s < E; s++) {
                    const int b = bin(s);
                    v[s] = scale(cmul(v[s], phasor<R>(Dturns[b], z)), ss[b]);
                }
            } else if (op == 9) {
                if (TmLayout<LOGN, LOGE>::ENABLED && tm != kNoTmem) {
                    TMS(tm).put(0, v);
                } else {
#pragma unroll
                    for (int s = 0; s < E; s++) scr0[bin(s)] = v[s];
                }
                load_u(v);
#pragma unroll
                for (int s = 0; s < E; s++) v[s] = cmul(v[s], phasor<R>(Dturns[bin(s)], z));
            } else if (op == 10) {
                if (TmLayout<LOGN, LOGE>::ENABLED && tm != kNoTmem) {
                    const TMS ts(tm);
                    ts.put(1, v);
#pragma unroll
                    for (int c = 0; c < TMS::CH; c++) {
                        C l[VPC];
                        ts.get(0, c, l);
#pragma unroll
                        for (int j = 0; j < VPC; j++) {
                            const int s = c * VPC + j;
                            const R I = g * abs2(v[s]);
                            const R Y = g * (l[j].im * v[s].re - l[j].re * v[s].im);
                            v[s] = mk(I, Y);
                        }
                    }
                } else {
#pragma unroll
                    for (int s = 0; s < E; s++) {
                        const int b = bin(s);
                        const C lt = scr0[b];
                        scr1[b] = v[s];
                        const R I = g * abs2(v[s]);
                        const R Y = g * (lt.im * v[s].re - lt.re * v[s].im);  // γ Im(λ u*)
                        v[s] = mk(I, Y);
                    }
                }
            } else if (op == 11) {
                // split the two real spectra (I and Y) with X[k] and conj(X[-k]);
                // Heff Î + i conj(Heff) Ŷ
                const C* __restrict__ Hp = Heff;
                split_pair_apply<R, LOGN, LOGE>(v, sm, [Hp](int b) { return Hp[b]; });
                inv = true;
            } else {  // op == 12
                // η = λ_t (2(1-fR) I + h∗I) - (1-fR) γ λ_t* u_t² + 2i (h̃⋆Y) u_t
                auto eta = [&](const C lt, const C ut, const C x) {
                    const R I = g * abs2(ut);
                    const R Rr = x.re * invn, Ri = x.im * invn;
                    const C t1 = scale(lt, R(2) * ofr * I + Rr);
                    const C t2 = scale(cmulc(cmul(ut, ut), lt), ofr * g);    // (1-fR)γ λ* u²
                    const C t3 = mk(-R(2) * Ri * ut.im, R(2) * Ri * ut.re);  // 2i Ri u
                    return t1 - t2 + t3;
                };
                if (TmLayout<LOGN, LOGE>::ENABLED && tm != kNoTmem) {
                    const TMS ts(tm);
#pragma unroll
                    for (int c = 0; c < TMS::CH; c++) {
                        C l[VPC], u[VPC];
                        ts.get2(c, l, u);
#pragma unroll
                        for (int j = 0; j < VPC; j++) v[c * VPC + j] = eta(l[j], u[j], v[c * VPC + j]);
                    }
                } else {
#pragma unroll
                    for (int s = 0; s < E; s++) {
                        const int b = bin(s);
                        v[s] = eta(scr0[b], scr1[b], v[s]);
                    }
                }
                inv = true;
            }
            if (inv) conj_all(v);
            block_fft<R, LOGN, LOGE>(v, sm, tw);
            if (inv) conj_all(v);
        }
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int b = bin(s);
            const C y = cmulc(v[s], phasor<R>(Dturns[b], z));  // e^{-iDz} x
            const R sc = adj ? invn : ss[b] * invn;
            v[s] = mk(-y.im * sc, y.re * sc);                      // i y (τ) / N
        }
    }

    // ---- stage helpers ---------------------------------------------------
    // logical stage i -> physical buffer; perm swaps stages 0 and 6 (FSAL)
    __device__ __forceinline__ static C* kp(void* const (&k)[7], int perm, int i) {
        int p = (perm && (i == 0 || i == 6)) ? 6 - i : i;
        return (C*)k[p];
    }

    // Stage combinations read the stage vectors stage-outer and point-inner:
    // each thread issues the loads of SC of its points for one stage
    // together, so SC loads are in flight per thread instead of one.  The
    // per-point summation order (stage 0 first) is unchanged.
    static constexpr int SC = E < 8 ? E : 8;                      // points per chunk
    static constexpr int SC7 = E < 8 ? E : (sizeof(R) == 8 ? 4 : 8);  // stage 7: two sums
    static_assert(E % SC == 0 && E % SC7 == 0, "chunks tile the thread's points");

    // v = ũ_n + dt Σ_{j<st} a[st][j] k_j   (FP64 accumulation)
    __device__ __forceinline__ void stage_input(int st, const double* u, void* const (&k)[7],
                                                int perm, double dt, IO v) {
#pragma unroll
        for (int s0 = 0; s0 < E; s0 += SC) {
            double ar[SC], ai[SC];
#pragma unroll
            for (int c = 0; c < SC; c++) ar[c] = ai[c] = 0.0;
#pragma unroll 1
            for (int j = 0; j < st; j++) {
                const C* __restrict__ kj = kp(k, perm, j);
                const double a = kT5a[st][j];
                C x[SC];
#pragma unroll
                for (int c = 0; c < SC; c++) x[c] = kj[bin(s0 + c)];
#pragma unroll
                for (int c = 0; c < SC; c++) {
                    ar[c] += a * (double)x[c].re;
                    ai[c] += a * (double)x[c].im;
                }
            }
#pragma unroll
            for (int c = 0; c < SC; c++) {
                const cx<double> un = ld2(u, bin(s0 + c));
                v[s0 + c] = mk((R)(un.re + dt * ar[c]), (R)(un.im + dt * ai[c]));
            }
        }
    }

    // stage 7 input = ũ_{n+1} (written to unew in FP64), partial error
    // dt Σ_{j<7} b̃_j k_j and the weights abstol + reltol max(|u_n|,|u_{n+1}|)
    __device__ __forceinline__ void stage7_input(const double* u, double* unew,
                                                 void* const (&k)[7], int perm, double dt,
                                                 double abstol, double reltol, IO v,
                                                 bool want_err) {
#pragma unroll
        for (int s0 = 0; s0 < E; s0 += SC7) {
            double ar[SC7], ai[SC7], er[SC7], ei[SC7];
#pragma unroll
            for (int c = 0; c < SC7; c++) ar[c] = ai[c] = er[c] = ei[c] = 0.0;
#pragma unroll 1
            for (int j = 0; j < 6; j++) {
                const C* __restrict__ kj = kp(k, perm, j);
                const double a = kT5a[6][j], bt = kT5bt[j];
                C x[SC7];
#pragma unroll
                for (int c = 0; c < SC7; c++) x[c] = kj[bin(s0 + c)];
#pragma unroll
                for (int c = 0; c < SC7; c++) {
                    ar[c] += a * (double)x[c].re;
                    ai[c] += a * (double)x[c].im;
                    er[c] += bt * (double)x[c].re;
                    ei[c] += bt * (double)x[c].im;
                }
            }
#pragma unroll
            for (int c = 0; c < SC7; c++) {
                const int b = bin(s0 + c);
                const cx<double> un = ld2(u, b);
                const cx<double> u1 = mk(un.re + dt * ar[c], un.im + dt * ai[c]);
                st2(unew, b, u1);
                if (want_err) {
                    st2(d.esv, b, mk(dt * er[c], dt * ei[c]));
                    const double m0 = sqrt(un.re * un.re + un.im * un.im);
                    const double m1 = sqrt(u1.re * u1.re + u1.im * u1.im);
                    d.skv[b] = abstol + fmax(m0, m1) * reltol;
                }
                v[s0 + c] = down<R>(u1);
            }
        }
    }

    // finish the error estimate with k7 (in v) -> EEst (block-uniform)
    __device__ __forceinline__ double error_norm(IO k7, double dt) {
        const double bt7 = kT5bt[6];
        double acc = 0.0;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int b = bin(s);
            const cx<double> e6 = ld2(d.esv, b);
            const double er = e6.re + dt * bt7 * (double)k7[s].re;
            const double ei = e6.im + dt * bt7 * (double)k7[s].im;
            const double w = d.skv[b];
            acc += (er * er + ei * ei) / (w * w);
        }
        const double tot = block_sum<T>(acc, red);
        return sqrt(tot / (double)N);
    }
};

// dense interpolant of a stored forward step (precision RF) at θ, into a
// field of precision R
template <typename RF, typename R, int LOGN, int LOGE>
__device__ __forceinline__ void interp_step(const SlotDesc& d, int slot, double dtn, double th,
                                            cx<R> (&w)[FftShape<LOGN, LOGE>::E]) {
    using S = FftShape<LOGN, LOGE>;
    constexpr int N = S::N, E = S::E, T = S::T;
    const cx<RF>* sg = (const cx<RF>*)d.seg + (size_t)slot * 5 * N;
    const double t2 = th * th, t3 = t2 * th, t4 = t3 * th;
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int b = threadIdx.x + T * s;
        const cx<RF> c0 = sg[b], c1 = sg[N + b], c2 = sg[2 * N + b], c3 = sg[3 * N + b],
                     c4 = sg[4 * N + b];
        const double xr = (double)c0.re + dtn * (th * (double)c1.re + t2 * (double)c2.re +
                                                 t3 * (double)c3.re + t4 * (double)c4.re);
        const double xi = (double)c0.im + dtn * (th * (double)c1.im + t2 * (double)c2.im +
                                                 t3 * (double)c3.im + t4 * (double)c4.im);
        w[s] = mk((R)xr, (R)xi);
    }
}

// PI controller: returns q and q11 (OrdinaryDiffEqCore stepsize_controller!)
__device__ __forceinline__ double pi_q(double EEst, double qold, double& q11) {
    if (EEst == 0.0) {
        q11 = 0.0;
        return 1.0 / kQmax;
    }
    q11 = pow(EEst, kBeta1);
    double q = q11 / pow(qold, kBeta2);
    q = q / kGamma;
    return fmax(1.0 / kQmax, fmin(1.0 / kQmin, q));
}

// Hairer initial step from the norms of the launch, f0 and the probe f1
// (OrdinaryDiffEqCore ode_determine_initdt; 5 = the method order).
__device__ __forceinline__ double initdt_first(double d0, double d1, double span) {
    double dt0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : (d0 / d1) / 100.0;
    return fmin(dt0, span);
}
__device__ __forceinline__ double initdt_final(double dt0, double d1, double d2, double nd,
                                               double dtmin, double span) {
    if (nd == 0.0) return fmax(dtmin, 100 * dt0);  // constant derivative over the probe
    const double mx = fmax(d1, d2);
    const double dt1 = mx <= 1e-15 ? fmax(1e-6, dt0 * 1e-3) : pow(10.0, -(2.0 + log10(mx)) / 5.0);
    return fmax(dtmin, fmin(fmin(100 * dt0, dt1), span));
}

// Forward field for the adjoint RHS: the dense interpolant of the stored step
// of the current segment that holds zz, or an FP64 field given directly.
template <typename RF, typename R, int LOGN, int LOGE>
struct SegLoader {
    static constexpr int E = FftShape<LOGN, LOGE>::E;
    const SlotDesc& d;
    int seg_lo, seg_hi;
    double zz;
    const double* direct;
    __device__ void operator()(cx<R> (&w)[E]) const {
        if (direct) {
#pragma unroll
            for (int s = 0; s < E; s++)
                w[s] = down<R>(ld2(direct, threadIdx.x + FftShape<LOGN, LOGE>::T * s));
            return;
        }
        // the last stored step of the segment starting at or before zz (the
        // logged step starts increase): a bisection, so a long segment costs
        // log2(length) dependent loads instead of one per step
        const double* lg = d.steplog;
        int n = seg_lo, hi = seg_hi - 1;
        while (n < hi) {
            const int mid = (n + hi + 1) >> 1;
            if (lg[2 * mid] <= zz) n = mid;
            else hi = mid - 1;
        }
        const double zn = lg[2 * n], dtn = lg[2 * n + 1];
        interp_step<RF, R, LOGN, LOGE>(d, n - seg_lo, dtn, (zz - zn) / dtn, w);
    }
};

// Out-of-line RHS evaluations.  The FFT-heavy bodies get the full register
// budget of the CTA instead of sharing it with the state machine's live
// values; the 2E-register field crosses the call through local memory.
template <typename R, int LOGN, int LOGE>
__device__ __noinline__ void rhs_fwd_call(const SlotDesc* d, void* sm, double* red, double z,
                                          FieldIO<cx<R>, LOGN, LOGE> vio,
                                          uint32_t tm = kNoTmem) {
    using Sol = SmSolver<R, LOGN, LOGE>;
    Sol S(*d, sm, red, tm);
    cx<R> v[Sol::E];
#pragma unroll
    for (int s = 0; s < Sol::E; s++) v[s] = vio[s];
    if constexpr (FieldIO<cx<R>, LOGN, LOGE>::SMEM) __syncthreads();
    S.rhs(false, z, v, [](cx<R>(&)[Sol::E]) {});
#pragma unroll
    for (int s = 0; s < Sol::E; s++) vio[s] = v[s];
}

template <typename RF, typename R, int LOGN, int LOGE>
__device__ __noinline__ void rhs_adj_call(const SlotDesc* d, void* sm, double* red, double z,
                                          FieldIO<cx<R>, LOGN, LOGE> vio, int seg_lo, int seg_hi,
                                          double zload, const double* ufwd,
                                          uint32_t tm = kNoTmem) {
    using Sol = SmSolver<R, LOGN, LOGE>;
    Sol S(*d, sm, red, tm);
    cx<R> v[Sol::E];
#pragma unroll
    for (int s = 0; s < Sol::E; s++) v[s] = vio[s];
    if constexpr (FieldIO<cx<R>, LOGN, LOGE>::SMEM) __syncthreads();
    SegLoader<RF, R, LOGN, LOGE> ld{*d, seg_lo, seg_hi, zload, ufwd};
    S.rhs(true, z, v, ld);
#pragma unroll
    for (int s = 0; s < Sol::E; s++) vio[s] = v[s];
}

// transform buffer (sized for the adjoint precision), 32 reduction doubles
// and the two twiddle tables
template <typename RA, int LOGN>
constexpr size_t smem_bytes() {
    return SmemPlan<RA, LOGN>::BYTES + 32 * sizeof(double) +
           sizeof(cx<float>) * Twiddles<float, LOGN>::SIZE +
           sizeof(cx<double>) * Twiddles<double, LOGN>::SIZE + 16;  // + the tensor-memory slot
}
// the shared-memory word tcgen05.alloc writes the tensor-memory address to
template <typename RA, int LOGN>
__device__ __forceinline__ uint32_t* tm_slot(unsigned char* smraw) {
    return reinterpret_cast<uint32_t*>(smraw + smem_bytes<RA, LOGN>() - 16);
}

// One RHS evaluation on one CTA (unit parity of the right-hand sides):
// in/ufwd/out are N complex doubles; forward in RF, adjoint in RA.
template <typename RF, typename RA, int LOGN, int LOGE>
__global__ void __launch_bounds__(FftShape<LOGN, LOGE>::T, 1)
    sm_rhs_kernel(const SlotDesc* __restrict__ d, int adjoint, double z,
                  const double* __restrict__ in, const double* __restrict__ ufwd,
                  double* __restrict__ out) {
    using S = FftShape<LOGN, LOGE>;
    extern __shared__ __align__(16) unsigned char smraw[];
    double* red = reinterpret_cast<double*>(smraw + SmemPlan<RA, LOGN>::BYTES);
    const uint32_t tm = tm_alloc<LOGN, LOGE>(tm_slot<RA, LOGN>(smraw));
    load_twiddles<LOGN>(*d, red);
    if (adjoint) {
        using IO = FieldIO<cx<RA>, LOGN, LOGE>;
        cx<RA> vl[IO::SMEM ? 1 : S::E];
        const IO v{IO::SMEM ? reinterpret_cast<cx<RA>*>(smraw) : vl};
#pragma unroll
        for (int s = 0; s < S::E; s++) v[s] = down<RA>(ld2(in, threadIdx.x + S::T * s));
        rhs_adj_call<RF, RA, LOGN, LOGE>(d, smraw, red, z, v, 0, 0, 0.0, ufwd, tm);
#pragma unroll
        for (int s = 0; s < S::E; s++) st2(out, threadIdx.x + S::T * s, up(v[s]));
    } else {
        using IO = FieldIO<cx<RF>, LOGN, LOGE>;
        cx<RF> vl[IO::SMEM ? 1 : S::E];
        const IO v{IO::SMEM ? reinterpret_cast<cx<RF>*>(smraw) : vl};
#pragma unroll
        for (int s = 0; s < S::E; s++) v[s] = down<RF>(ld2(in, threadIdx.x + S::T * s));
        rhs_fwd_call<RF, LOGN, LOGE>(d, smraw, red, z, v, tm);
#pragma unroll
        for (int s = 0; s < S::E; s++) st2(out, threadIdx.x + S::T * s, up(v[s]));
    }
    tm_free<LOGN, LOGE>(tm);
}

// Steps [lo, hi) of the current sub-segment: the segment of checkpoint seg
// (ck_stride steps) is replayed and integrated backward in sub-segments of at
// most seg_cap steps, last first.  Each sub-segment replays the segment from
// its checkpoint; the steps before the sub-segment are recomputed without
// storing their interpolant, so a solve of any length fits the K checkpoints
// and the seg_cap-step interpolant buffer (at the cost of recomputation that
// grows with ck_stride / seg_cap) instead of failing for capacity.
// (Shared by the single-mode and the multimode steppers: Desc / State are
// SlotDesc / SlotState or MmDesc / MmState.)
struct SubSeg {
    int seg_lo, seg_hi, lo, hi;
};
template <class Desc, class State>
__device__ __forceinline__ SubSeg sub_segment(const Desc& d, const State& st) {
    SubSeg r;
    if (st.dense) {  // the forward kept the interpolant of every step: one range
        r.seg_lo = r.lo = 0;
        r.seg_hi = r.hi = st.nsteps;
        return r;
    }
    r.seg_lo = st.seg * st.ck_stride;
    r.seg_hi = min(r.seg_lo + st.ck_stride, st.nsteps);
    r.lo = r.seg_lo + st.sub * d.seg_cap;
    r.hi = min(r.lo + d.seg_cap, r.seg_hi);
    return r;
}
// index of the last sub-segment of segment seg
template <class Desc, class State>
__device__ __forceinline__ int last_sub(const Desc& d, const State& st, int seg) {
    const int lo = seg * st.ck_stride, hi = min(lo + st.ck_stride, st.nsteps);
    return (hi - lo - 1) / d.seg_cap;
}

// Dense interpolant of an accepted step into sg (5 fields): c0 = ũ_n,
// c_p = Σ_i r_ip k_i (Tsit5's free 4th-order interpolant), read stage-outer
// over chunks of 4 points per thread as in stage_input.
template <typename RF, int LOGN, int LOGE>
__device__ __forceinline__ void store_interp(const SlotDesc& d, const double* u, int kperm,
                                             cx<RF>* sg) {
    using S = FftShape<LOGN, LOGE>;
    using Sol = SmSolver<RF, LOGN, LOGE>;
    using CF = cx<RF>;
    constexpr int N = S::N, E = S::E;
    constexpr int RC = E < 4 ? E : 4;
    static_assert(E % RC == 0, "chunks tile the thread's points");
#pragma unroll
    for (int s0 = 0; s0 < E; s0 += RC) {
        double cr[RC][4], ci[RC][4];
#pragma unroll
        for (int c = 0; c < RC; c++)
#pragma unroll
            for (int q = 0; q < 4; q++) cr[c][q] = ci[c][q] = 0.0;
#pragma unroll 1
        for (int i = 0; i < 7; i++) {
            const CF* __restrict__ kv = Sol::kp(d.kf, kperm, i);
            CF x[RC];
#pragma unroll
            for (int c = 0; c < RC; c++) x[c] = kv[Sol::bin(s0 + c)];
#pragma unroll
            for (int c = 0; c < RC; c++)
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    cr[c][q] += kT5r[i][q] * (double)x[c].re;
                    ci[c][q] += kT5r[i][q] * (double)x[c].im;
                }
        }
#pragma unroll
        for (int c = 0; c < RC; c++) {
            const int b = Sol::bin(s0 + c);
            sg[b] = down<RF>(ld2(u, b));
#pragma unroll
            for (int q = 0; q < 4; q++) sg[(q + 1) * N + b] = mk((RF)cr[c][q], (RF)ci[c][q]);
        }
    }
}

// Checked build (-DFL_CHECKED): before each step of the state machine, the
// indices a step will use -- stage, buffer parities, the step count against
// the step log, the checkpoint segment and sub-segment against the
// checkpoint slots and the interpolant buffer, the save position -- are
// checked against their buffers.  A violation ends the slot with ST_CHECK
// (FL_ECHECK) before any access, instead of trapping.  The default build
// compiles the check away.  Shared by both steppers (SlotDesc / SlotState,
// MmDesc / MmState).
template <class Desc, class State>
__device__ __forceinline__ bool state_in_bounds(const Desc& d, const State& st) {
    bool ok = st.stage >= 0 && st.stage <= 6 && (st.cur | st.kperm | st.acur | st.akperm) >= 0 &&
              (st.cur | st.kperm | st.acur | st.akperm) <= 1 && st.save_idx >= 0 &&
              st.save_idx <= d.nsave && st.nsteps >= 0 &&
              (d.step_cap == 0 || st.nsteps <= d.step_cap);
    const int ph = st.phase;
    if (ok && (ph == PH_REC || ph == PH_ADJ_INIT || ph == PH_ADJ)) {
        const SubSeg sb = sub_segment(d, st);
        // a replay has steps left in its sub-segment; the adjoint follows a
        // finished replay (rec_pos at the sub-segment's end)
        const int rec_end = sb.seg_lo + st.rec_pos;
        ok = d.step_cap > 0 && st.nsteps >= 1 && sb.lo >= 0 && sb.lo < sb.hi &&
             sb.hi <= st.nsteps && sb.hi - sb.lo <= d.seg_cap && st.rec_pos >= 0 &&
             (st.dense || (st.seg >= 0 && st.seg < d.ck_cap && st.ck_stride >= 1 &&
                           (ph == PH_REC ? rec_end < sb.hi : rec_end <= sb.hi)));
    }
    return ok;
}

template <typename RF, int LOGN, int LOGE>
__device__ __forceinline__ void restore_checkpoint(const SlotDesc& d, int seg, SlotState& st) {
    using S = FftShape<LOGN, LOGE>;
    constexpr int N = S::N, E = S::E, T = S::T;
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int b = threadIdx.x + T * s;
        reinterpret_cast<double2*>(d.u[0])[b] =
            reinterpret_cast<const double2*>(d.ck_u)[(size_t)seg * N + b];
        ((cx<RF>*)d.kf[0])[b] = ((const cx<RF>*)d.ck_k1)[(size_t)seg * N + b];
    }
    st.cur = 0;
    st.kperm = 0;
    st.rec_pos = 0;
    st.stage = 0;
}

// Hairer initial step, part 1 (after f0): stores f0 as the FSAL derivative,
// returns the probe step dt0 (> 0) or, when no probe is needed, -dtinit.
template <typename K, int LOGN, int LOGE>
__device__ __forceinline__ double init_after_f0(const double* x0, cx<K>* k1,
                                                FieldIO<cx<K>, LOGN, LOGE> v,
                                                double at, double rt, double L, double dtmin,
                                                double* red, double& d1_out) {
    using S = FftShape<LOGN, LOGE>;
    constexpr int N = S::N, E = S::E, T = S::T;
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int b = threadIdx.x + T * s;
        k1[b] = v[s];
        const cx<double> x = ld2(x0, b);
        const double ax = sqrt(x.re * x.re + x.im * x.im);
        const double sk = at + ax * rt;
        s0 += (ax / sk) * (ax / sk);
        const double af = sqrt(abs2(up(v[s])));
        s1 += (af / sk) * (af / sk);
    }
    const double d0 = sqrt(block_sum<T>(s0, red) / N);
    const double d1 = sqrt(block_sum<T>(s1, red) / N);
    d1_out = d1;
    const double dt0 = initdt_first(d0, d1, L);
    if (!isfinite(d1)) return -dtmin;
    if (dt0 < 10 * kEps) return -fmax(1e-6, dtmin);
    return dt0;
}

// Hairer initial step, part 2 (after the probe f1 at x0 ± dt0 f0)
template <typename K, int LOGN, int LOGE>
__device__ __forceinline__ double init_after_f1(const double* x0, const cx<K>* k1,
                                                FieldIO<cx<K>, LOGN, LOGE> v,
                                                double at, double rt, double dt0, double d1,
                                                double L, double dtmin, double* red) {
    using S = FftShape<LOGN, LOGE>;
    constexpr int N = S::N, E = S::E, T = S::T;
    double s2 = 0.0, ndiff = 0.0;
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int b = threadIdx.x + T * s;
        const cx<double> x = ld2(x0, b);
        const double sk = at + sqrt(x.re * x.re + x.im * x.im) * rt;
        const cx<K> f0 = k1[b];
        const double dr = (double)v[s].re - (double)f0.re;
        const double di = (double)v[s].im - (double)f0.im;
        s2 += (dr * dr + di * di) / (sk * sk);
        ndiff += (dr != 0.0 || di != 0.0) ? 1.0 : 0.0;
    }
    const double d2 = sqrt(block_sum<T>(s2, red) / N) / dt0;
    const double nd = block_sum<T>(ndiff, red);
    return initdt_final(dt0, d1, d2, nd, dtmin, L);
}

// The state machine.  Each loop iteration performs at most one RHS
// evaluation (forward in RF, adjoint in RA) plus the bookkeeping around it,
// so the FFT code exists once per precision in the kernel.
template <typename RF, typename RA, int LOGN, int LOGE>
__global__ void __launch_bounds__(FftShape<LOGN, LOGE>::T, 1)
    sm_advance_kernel(const SlotDesc* __restrict__ descs, SlotState* __restrict__ states,
                      const int* __restrict__ active, int max_evals) {
    using SolF = SmSolver<RF, LOGN, LOGE>;
    using SolA = SmSolver<RA, LOGN, LOGE>;
    using CF = cx<RF>;
    using CA = cx<RA>;
    constexpr int N = SolF::N, E = SolF::E, T = SolF::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    double* red = reinterpret_cast<double*>(smraw + SmemPlan<RA, LOGN>::BYTES);

    const int slot = active[blockIdx.x];
    const SlotDesc& d = descs[slot];
    const uint32_t tm = tm_alloc<LOGN, LOGE>(tm_slot<RA, LOGN>(smraw));
    load_twiddles<LOGN>(d, red);
    SlotState st = states[slot];  // block-uniform copy
    SolF SF(d, smraw, red);
    SolA SA(d, smraw, red);
    const int tid = threadIdx.x;
    const double L = d.L, dtmin = kEps * L;
    using IOF = FieldIO<CF, LOGN, LOGE>;
    using IOA = FieldIO<CA, LOGN, LOGE>;
    CF vfl[IOF::SMEM ? 1 : E];  // local-memory field (Nt = 2^14 only)
    CA val[IOA::SMEM ? 1 : E];
    const IOF vf{IOF::SMEM ? reinterpret_cast<CF*>(smraw) : vfl};
    const IOA va{IOA::SMEM ? reinterpret_cast<CA*>(smraw) : val};
    int evals = 0;

    while (st.phase != PH_DONE && evals < max_evals) {
#ifdef FL_CHECKED
        if (!state_in_bounds(d, st)) {
            st.status = ST_CHECK;
            st.phase = PH_DONE;
            continue;
        }
#endif
        // ------------------------------------------------ phases without an RHS
        if (st.phase == PH_SEED) {
            // terminal seed λ̃(L) (interaction frame) into lam[0]
            const double* uf = d.u[st.cur];
            double* lam = d.lam[0];
            if (d.mode == MODE_BAND_GRADIENT) {
                // Band objective (physics_helpers.jl:222-232).  With one mode
                // the fundamental-mode and worst-mode objectives are the same
                // (:234-286: one active mode, log-sum-exp = its fraction,
                // weight 1).  The peak objective (:288-302) puts the strongest
                // in-band bin (lowest index among equals) in place of the band.
                const bool peak = d.objective == OBJ_RAMAN_PEAK;
                double et = 0.0, eb = 0.0, emax = -1.0;
#pragma unroll
                for (int s = 0; s < E; s++) {
                    const int b = SolF::bin(s);
                    const double e = energy(ld2(uf, b));
                    et += e;
                    if (d.mask[b]) {
                        eb += e;
                        emax = fmax(emax, e);
                    }
                }
                const double tot = block_sum<T>(et, red);
                double band = block_sum<T>(eb, red);
                int pk = -1;
                if (peak) {
                    band = block_max<T>(emax, red);
                    // lowest index as the largest key N - b (block_max folds from 0)
                    double key = 0.0;
#pragma unroll
                    for (int s = 0; s < E; s++) {
                        const int b = SolF::bin(s);
                        if (d.mask[b] && energy(ld2(uf, b)) == band) key = fmax(key, (double)(N - b));
                    }
                    pk = N - (int)block_max<T>(key, red);
                }
                const double cost = band / tot;
                double sc = 1.0 / tot;
                st.J = cost;
                if (d.log_cost) {  // physics_helpers.jl:320-326
                    st.J = 10.0 * log10(fmax(cost, 1e-15));
                    sc *= cost <= 1e-15 ? 0.0 : 10.0 / (log(10.0) * cost);
                }
                // e^{-iDL} (u_L (sel - J)/E) = ũ(L) (sel - J)/E, sel the band or peak bin
#pragma unroll
                for (int s = 0; s < E; s++) {
                    const int b = SolF::bin(s);
                    const cx<double> x = ld2(uf, b);
                    const double sel = peak ? (b == pk ? 1.0 : 0.0) : (d.mask[b] ? 1.0 : 0.0);
                    const double f = (sel - cost) * sc;
                    st2(lam, b, mk(x.re * f, x.im * f));
                }
            } else {
                st.J = 0.0;
#pragma unroll
                for (int s = 0; s < E; s++) {
                    const int b = SolF::bin(s);
                    const cx<double> x = ld2(d.lamL, b);
                    const cx<double> p = phasor<double>(d.Dturns[b], L);
                    st2(lam, b, mk(x.re * p.re + x.im * p.im, x.im * p.re - x.re * p.im));
                }
            }
            double mx = 0.0;
            bool finite = true;
#pragma unroll
            for (int s = 0; s < E; s++) {
                const cx<double> x = ld2(lam, SolF::bin(s));
                const double a = sqrt(x.re * x.re + x.im * x.im);
                if (!isfinite(a)) finite = false;
                mx = fmax(mx, a);
            }
            const double scl = block_max<T>(finite ? mx : INFINITY, red);
            if (!isfinite(scl)) {
                st.status = ST_NONFINITE;
                st.phase = PH_DONE;
                continue;
            }
            st.abstol_adj = scl == 0.0 ? d.abstol : d.abstol * scl;  // sensitivity_disp_mmf.jl:324-325
            st.acur = 0;
            st.akperm = 0;
            st.a_naccept = st.a_nreject = st.a_nf = st.a_iters = 0;
            st.nrec = 0;
            // every step's interpolant is in the buffer when the forward fit it
            // (kept by the forward; an earlier adjoint of this solve then did
            // not overwrite it)
            st.dense = st.nsteps <= d.seg_cap ? 1 : 0;
            if (st.dense) {
                st.seg = 0;
                st.sub = 0;
                st.phase = PH_ADJ_INIT;
                continue;
            }
            st.seg = (st.nsteps + st.ck_stride - 1) / st.ck_stride - 1;
            st.sub = last_sub(d, st, st.seg);
            restore_checkpoint<RF, LOGN, LOGE>(d, st.seg, st);
            st.phase = PH_REC;
            continue;
        }
        if (st.phase == PH_FINAL) {
            // λ(0) = λ̃(0); ∂J/∂φ = 2 Re(conj(λ0) i u_shaped) (physics_models.jl:1042)
            const double* lam = d.lam[st.acur];
#pragma unroll
            for (int s = 0; s < E; s++) {
                const int b = SolF::bin(s);
                const cx<double> l = ld2(lam, b);
                if (d.lam0_out) st2(d.lam0_out, b, l);
                if (d.grad_out) {
                    const cx<double> us = ld2(d.u0, b);
                    d.grad_out[b] = 2.0 * (l.im * us.re - l.re * us.im);
                }
            }
            st.phase = PH_DONE;
            continue;
        }

        // ------------------------------------------------ build the stage input
        const bool adj = st.phase == PH_ADJ_INIT || st.phase == PH_ADJ;
        double ze = 0.0, zload = 0.0;
        if (st.phase == PH_FWD_INIT) {
            const CF* k1 = (const CF*)d.kf[0];
#pragma unroll
            for (int s = 0; s < E; s++) {
                const int b = SolF::bin(s);
                const cx<double> x = ld2(d.u0, b);
                if (st.stage == 0) {
                    st2(d.u[0], b, x);
                    vf[s] = down<RF>(x);
                } else {
                    const CF f0 = k1[b];
                    vf[s] = mk((RF)(x.re + st.cdt * (double)f0.re),
                               (RF)(x.im + st.cdt * (double)f0.im));
                }
            }
            ze = st.stage == 0 ? 0.0 : st.cdt;
        } else if (st.phase == PH_FWD || st.phase == PH_REC) {
            if (st.stage == 0) {
                if (st.phase == PH_REC) {
                    const int n = st.seg * st.ck_stride + st.rec_pos;
                    st.cz = d.steplog[2 * n];
                    st.cdt = d.steplog[2 * n + 1];
                } else {
                    if (++st.iters > d.max_iters) {
                        st.status = ST_MAXITERS;
                        st.phase = PH_DONE;
                        continue;
                    }
                    // fix_dt_at_bounds!, modify_dt_for_tstops!
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
            const double* u = d.u[st.cur];
            if (st.stage < 6)
                SF.stage_input(st.stage, u, d.kf, st.kperm, st.cdt, vf);
            else
                SF.stage7_input(u, d.u[st.cur ^ 1], d.kf, st.kperm, st.cdt, d.abstol, d.reltol,
                                vf, st.phase == PH_FWD);
            ze = st.cz + kT5c[st.stage] * st.cdt;
        } else if (st.phase == PH_ADJ_INIT) {
            const double* lam = d.lam[0];
            const CA* k1 = (const CA*)d.ka[0];
#pragma unroll
            for (int s = 0; s < E; s++) {
                const int b = SolF::bin(s);
                const cx<double> x = ld2(lam, b);
                if (st.stage == 0) {
                    va[s] = down<RA>(x);
                } else {
                    const CA f0 = k1[b];
                    va[s] = mk((RA)(x.re - st.cdt * (double)f0.re),
                               (RA)(x.im - st.cdt * (double)f0.im));
                }
            }
            ze = st.stage == 0 ? L : L - st.cdt;
            zload = st.stage == 0 ? L : fmax(ze, d.steplog[2 * sub_segment(d, st).lo]);
        } else {  // PH_ADJ
            const double zlo = d.steplog[2 * sub_segment(d, st).lo];
            if (st.stage == 0) {
                if (++st.a_iters > d.max_iters) {
                    st.status = ST_MAXITERS;
                    st.phase = PH_DONE;
                    continue;
                }
                // Segment starts are stopping points of this implementation only
                // (the reference integrates the adjoint without them), so they
                // are made transparent to the controller: no sliver step before
                // one (the last two steps are split evenly) and the proposal
                // from before the clip is restored after it.
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
            const double* lam = d.lam[st.acur];
            if (st.stage < 6)
                SA.stage_input(st.stage, lam, d.ka, st.akperm, st.cdt, va);
            else
                SA.stage7_input(lam, d.lam[st.acur ^ 1], d.ka, st.akperm, st.cdt, st.abstol_adj,
                                d.reltol, va, true);
            ze = zload = st.cz + kT5c[st.stage] * st.cdt;
        }

        // ------------------------------------------------ one RHS evaluation
        if (adj) {
            const SubSeg sb = sub_segment(d, st);
            rhs_adj_call<RF, RA, LOGN, LOGE>(&d, smraw, red, ze, va, sb.lo, sb.hi, zload,
                                             nullptr, tm);
        } else {
            rhs_fwd_call<RF, LOGN, LOGE>(&d, smraw, red, ze, vf, tm);
        }
        evals++;

        // ------------------------------------------------ consume the derivative
        if (st.phase == PH_FWD_INIT || st.phase == PH_ADJ_INIT) {
            const bool fw = st.phase == PH_FWD_INIT;
            if (st.stage == 0) {
                double d1;
                const double r = fw ? init_after_f0<RF, LOGN, LOGE>(d.u0, (CF*)d.kf[0], vf,
                                                                    d.abstol, d.reltol, L, dtmin,
                                                                    red, d1)
                                    : init_after_f0<RA, LOGN, LOGE>(d.lam[0], (CA*)d.ka[0], va,
                                                                    st.abstol_adj, d.reltol, L,
                                                                    dtmin, red, d1);
                if (r > 0.0) {  // probe step
                    st.cdt = r;
                    st.cz = d1;
                    st.stage = 1;
                    continue;
                }
                st.cdt = -r;
            } else {
                st.cdt = fw ? init_after_f1<RF, LOGN, LOGE>(d.u0, (const CF*)d.kf[0], vf,
                                                            d.abstol, d.reltol, st.cdt, st.cz, L,
                                                            dtmin, red)
                            : init_after_f1<RA, LOGN, LOGE>(d.lam[0], (const CA*)d.ka[0], va,
                                                            st.abstol_adj, d.reltol, st.cdt,
                                                            st.cz, L, dtmin, red);
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
                st.naccept = st.nreject = st.iters = 0;
                st.nf = 3;
                if (d.ck_cap > 0) {
                    const CF* k1 = (const CF*)d.kf[0];
#pragma unroll
                    for (int s = 0; s < E; s++) {
                        const int b = SolF::bin(s);
                        reinterpret_cast<double2*>(d.ck_u)[b] =
                            reinterpret_cast<const double2*>(d.u0)[b];
                        ((CF*)d.ck_k1)[b] = k1[b];
                    }
                }
                st.save_idx = 0;
                while (st.save_idx < d.nsave && d.zsave[st.save_idx] == 0.0) {
                    double* o = d.save_out + (size_t)st.save_idx * 2 * N;
#pragma unroll
                    for (int s = 0; s < E; s++) st2(o, SolF::bin(s), ld2(d.u0, SolF::bin(s)));
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
            continue;
        }

        if (st.phase == PH_FWD || st.phase == PH_REC) {
            const bool rec = st.phase == PH_REC;
            CF* ko = SolF::kp(d.kf, st.kperm, st.stage);
#pragma unroll
            for (int s = 0; s < E; s++) ko[SolF::bin(s)] = vf[s];
            if (st.stage < 6) {
                st.stage++;
                continue;
            }
            st.stage = 0;
            const double z = st.cz, dt = st.cdt;
            const double* u = d.u[st.cur];
            if (rec) {
                // interpolant of this step, kept only for the steps of the
                // current sub-segment
                const SubSeg sb = sub_segment(d, st);
                const int n = sb.seg_lo + st.rec_pos;
                if (n >= sb.lo)
                    store_interp<RF, LOGN, LOGE>(d, u, st.kperm,
                                                 (CF*)d.seg + (size_t)(n - sb.lo) * 5 * N);
                st.cur ^= 1;
                st.kperm ^= 1;
                st.rec_pos++;
                st.nrec++;
                if (n + 1 >= sb.hi) st.phase = st.a_nf == 0 ? PH_ADJ_INIT : PH_ADJ;
                continue;
            }
            const double EEst = SF.error_norm(vf, dt);
            if (!isfinite(EEst)) {
                st.status = ST_NONFINITE;
                st.phase = PH_DONE;
                continue;
            }
            double q11;
            const double q = pi_q(EEst, st.qold, q11);
            st.nf += 6;
            if (EEst > 1.0) {
                st.nreject++;
                st.dt = dt / fmin(1.0 / kQmin, q11 / kGamma);
                continue;
            }
            st.naccept++;
            if (d.step_cap > 0) {  // step_cap 0: forward only, nothing kept for an adjoint
                if (st.nsteps >= d.step_cap) {
                    st.status = ST_CAPACITY;
                    st.phase = PH_DONE;
                    continue;
                }
                if (tid == 0) {
                    d.steplog[2 * st.nsteps] = z;
                    d.steplog[2 * st.nsteps + 1] = dt;
                }
                // while the solve fits the interpolant buffer, keep each
                // step's interpolant now: the adjoint then needs no recompute
                if (st.nsteps < d.seg_cap)
                    store_interp<RF, LOGN, LOGE>(d, u, st.kperm,
                                                 (CF*)d.seg + (size_t)st.nsteps * 5 * N);
            }
            double znew = z + dt;
            if (fabs(znew - L) < 100.0 * kEps * fmax(z, L)) znew = L;  // snap to the tstop
            // save positions in (z, znew) and on an interior step end: dense
            // output (positions at L take the final state below)
            while (st.save_idx < d.nsave && d.zsave[st.save_idx] > z &&
                   (d.zsave[st.save_idx] < znew || (d.zsave[st.save_idx] == znew && znew < L))) {
                const double zs = d.zsave[st.save_idx];
                const double th = (zs - z) / dt;
                double* o = d.save_out + (size_t)st.save_idx * 2 * N;
#pragma unroll
                for (int s = 0; s < E; s++) {
                    const int b = SolF::bin(s);
                    double xr = 0.0, xi = 0.0;
                    for (int i = 0; i < 7; i++) {
                        double bi = 0.0, tp = th;
                        for (int qq = 0; qq < 4; qq++) {
                            bi += kT5r[i][qq] * tp;
                            tp *= th;
                        }
                        const CF ki = SolF::kp(d.kf, st.kperm, i)[b];
                        xr += bi * (double)ki.re;
                        xi += bi * (double)ki.im;
                    }
                    const cx<double> un = ld2(u, b);
                    const cx<double> x = mk(un.re + dt * xr, un.im + dt * xi);
                    const cx<double> p = phasor<double>(d.Dturns[b], zs);
                    st2(o, b, mk(x.re * p.re - x.im * p.im, x.re * p.im + x.im * p.re));
                }
                st.save_idx++;
            }
            st.nsteps++;
            st.z = znew;
            st.cur ^= 1;
            st.kperm ^= 1;
            st.qold = fmax(EEst, kQoldInit);
            st.dt = fmin(fmax((q == 1.0) ? dt : dt / q, dtmin), L);
            // z-checkpoints with thinning: K slots at steps j*stride
            if (d.ck_cap > 0 && (st.nsteps % st.ck_stride) == 0) {
                int slotc = st.nsteps / st.ck_stride;
                if (slotc >= d.ck_cap) {
                    for (int j = 1; j < d.ck_cap / 2; j++) {
#pragma unroll
                        for (int s = 0; s < E; s++) {
                            const int b = SolF::bin(s);
                            reinterpret_cast<double2*>(d.ck_u)[(size_t)j * N + b] =
                                reinterpret_cast<double2*>(d.ck_u)[(size_t)2 * j * N + b];
                            ((CF*)d.ck_k1)[(size_t)j * N + b] =
                                ((CF*)d.ck_k1)[(size_t)2 * j * N + b];
                        }
                    }
                    st.ck_stride *= 2;
                    slotc = st.nsteps / st.ck_stride;
                }
#ifdef FL_CHECKED
                if (slotc < 0 || slotc >= d.ck_cap) {
                    st.status = ST_CHECK;
                    st.phase = PH_DONE;
                    continue;
                }
#endif
                const double* un = d.u[st.cur];
                const CF* k1 = SolF::kp(d.kf, st.kperm, 0);
#pragma unroll
                for (int s = 0; s < E; s++) {
                    const int b = SolF::bin(s);
                    reinterpret_cast<double2*>(d.ck_u)[(size_t)slotc * N + b] =
                        reinterpret_cast<const double2*>(un)[b];
                    ((CF*)d.ck_k1)[(size_t)slotc * N + b] = k1[b];
                }
            }
            if (st.z == L) {
                const double* uf = d.u[st.cur];
#pragma unroll
                for (int s = 0; s < E; s++) {
                    const int b = SolF::bin(s);
                    const cx<double> x = ld2(uf, b);
                    const cx<double> p = phasor<double>(d.Dturns[b], L);
                    const cx<double> y = mk(x.re * p.re - x.im * p.im, x.re * p.im + x.im * p.re);
                    for (int si = st.save_idx; si < d.nsave; si++)
                        st2(d.save_out + (size_t)si * 2 * N, b, y);
                    if (d.uL_out) st2(d.uL_out, b, y);
                }
                st.save_idx = d.nsave;
                st.phase = d.mode == MODE_FORWARD ? PH_DONE : PH_SEED;
            }
            continue;
        }

        // PH_ADJ
        {
            CA* ko = SolA::kp(d.ka, st.akperm, st.stage);
#pragma unroll
            for (int s = 0; s < E; s++) ko[SolF::bin(s)] = va[s];
            if (st.stage < 6) {
                st.stage++;
                continue;
            }
            st.stage = 0;
            const double z = st.cz, dt = st.cdt;
            const double zlo = d.steplog[2 * sub_segment(d, st).lo];
            const double EEst = SA.error_norm(va, dt);
            if (!isfinite(EEst)) {
                st.status = ST_NONFINITE;
                st.phase = PH_DONE;
                continue;
            }
            double q11;
            const double q = pi_q(EEst, st.aqold, q11);
            st.a_nf += 6;
            if (EEst > 1.0) {
                st.a_nreject++;
                st.adt = st.adt / fmin(1.0 / kQmin, q11 / kGamma);
                continue;
            }
            st.a_naccept++;
            double znew = z + dt;
            if (fabs(znew - zlo) < 100.0 * kEps * fmax(z, zlo)) znew = zlo;
            st.az = znew;
            st.acur ^= 1;
            st.akperm ^= 1;
            st.aqold = fmax(EEst, kQoldInit);
            const double adt = -dt;
            double dtn = fmin(fmax((q == 1.0) ? adt : adt / q, dtmin), L);
            if (adt < st.aprop) dtn = fmax(dtn, st.aprop);  // shortened for a segment start
            st.adt = -dtn;
            if (st.az == zlo) {
                if (st.sub > 0) {  // the previous sub-segment of this segment
                    st.sub--;
                    restore_checkpoint<RF, LOGN, LOGE>(d, st.seg, st);
                    st.phase = PH_REC;
                } else if (st.seg == 0) {
                    st.phase = PH_FINAL;
                } else {
                    st.seg--;
                    st.sub = last_sub(d, st, st.seg);
                    restore_checkpoint<RF, LOGN, LOGE>(d, st.seg, st);
                    st.phase = PH_REC;
                }
            }
        }
    }
    __syncthreads();
    if (tid == 0) states[slot] = st;
    tm_free<LOGN, LOGE>(tm);
}

}  // namespace fl
