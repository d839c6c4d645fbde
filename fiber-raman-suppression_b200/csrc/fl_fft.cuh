// fl_fft.cuh -- block-wide Stockham FFT for one CTA, sm_100a.
//
// A length-N transform (N = T*E) is held E elements per thread: thread t owns
// the samples/bins {t + s*T : s in [0, E)}.  The transform runs as radix-E
// Stockham passes (plus one smaller-radix pass when log2 E does not divide
// log2 N).  Inputs of the first pass and outputs of the last pass sit in the
// same registers with the same ownership, so a forward transform, a pointwise
// operation and an inverse transform never need a reorder pass; only the
// passes in between exchange data through one padded shared-memory buffer.
//
// Conventions match FFTW as used by the reference: the forward transform is
// unnormalised with exponent sign -1; the "inverse" here is the unnormalised
// sign +1 transform (callers fold the 1/N of ifft into their pointwise step).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fl {

template <typename R>
struct __align__(2 * sizeof(R)) cx {
    R re, im;
};

template <typename R>
__device__ __forceinline__ cx<R> mk(R a, R b) {
    cx<R> z;
    z.re = a;
    z.im = b;
    return z;
}
template <typename R>
__device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b) { return mk(a.re + b.re, a.im + b.im); }
template <typename R>
__device__ __forceinline__ cx<R> operator-(cx<R> a, cx<R> b) { return mk(a.re - b.re, a.im - b.im); }
template <typename R>
__device__ __forceinline__ cx<R> cmul(cx<R> a, cx<R> b) {
    return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename R>
__device__ __forceinline__ cx<R> cmulc(cx<R> a, cx<R> b) {  // a * conj(b)
    return mk(a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im);
}
template <typename R>
__device__ __forceinline__ cx<R> scale(cx<R> a, R s) { return mk(a.re * s, a.im * s); }
template <typename R>
__device__ __forceinline__ cx<R> conjc(cx<R> a) { return mk(a.re, -a.im); }
template <typename R>
__device__ __forceinline__ R abs2(cx<R> a) { return a.re * a.re + a.im * a.im; }
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename R>
__device__ __forceinline__ cx<R> rot90(cx<R> a) {
    return INV ? mk(-a.im, a.re) : mk(a.im, -a.re);
}

// padded shared-memory index: one pad element every 16 keeps the stride-16
// writes of the first pass conflict-free for 8- and 16-byte elements
__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded_len(int n) { return n + (n >> 4); }

// exp(-2 pi i k/32) for k = 0..15: (cos, -sin) at multiples of pi/16
// (literal values of the elementary constants).
template <typename R>
__device__ __forceinline__ cx<R> w32(int k) {
    constexpr double C[16] = {1.0,
                              0.98078528040323043058,
                              0.92387953251128673848,
                              0.83146961230254523567,
                              0.70710678118654752440,
                              0.55557023301960222474,
                              0.38268343236508977173,
                              0.19509032201612826785,
                              0.0,
                              -0.19509032201612826785,
                              -0.38268343236508977173,
                              -0.55557023301960222474,
                              -0.70710678118654752440,
                              -0.83146961230254523567,
                              -0.92387953251128673848,
                              -0.98078528040323043058};
    // sin(pi k/16) = cos(pi (8 - k)/16) for k <= 8, = cos(pi (k - 8)/16) beyond
    const double c = C[k];
    const double s = k <= 8 ? C[8 - k] : C[k - 8];
    return mk<R>(R(c), R(-s));
}

// multiply by exp(-+2 pi i k / 32) with the trivial cases special-cased
template <bool INV, typename R>
__device__ __forceinline__ cx<R> tw32(cx<R> a, int k) {
    if (k == 0) return a;
    if (k == 8) return rot90<INV>(a);
    cx<R> w = w32<R>(k);
    if (INV) w.im = -w.im;
    return cmul(a, w);
}

// In-register radix-RAD DFT on a[base + STRIDE*r], r in [0, RAD):
// radix-2 decimation-in-frequency stages, output de-scrambled by register
// renaming (bit reversal of a compile-time index).  Loops are fully unrolled
// so every index is a compile-time constant.
template <int RAD, bool INV, int STRIDE, typename R, int E>
__device__ __forceinline__ void dft_inreg(cx<R> (&a)[E], const int base) {
    static_assert(RAD == 1 || RAD == 2 || RAD == 4 || RAD == 8 || RAD == 16 || RAD == 32,
                  "radix");
    if constexpr (RAD >= 2) {
#pragma unroll
        for (int half = RAD / 2; half >= 1; half >>= 1) {
#pragma unroll
            for (int blk = 0; blk < RAD; blk += 2 * half) {
#pragma unroll
                for (int j = 0; j < half; j++) {
                    cx<R> u = a[base + STRIDE * (blk + j)];
                    cx<R> v = a[base + STRIDE * (blk + j + half)];
                    a[base + STRIDE * (blk + j)] = u + v;
                    // twiddle exp(-2 pi i j / (2 half)) = w32^(j * 32 / (2 half))
                    a[base + STRIDE * (blk + j + half)] = tw32<INV>(u - v, j * (32 / (2 * half)));
                }
            }
        }
        constexpr int LG = RAD == 2 ? 1 : RAD == 4 ? 2 : RAD == 8 ? 3 : RAD == 16 ? 4 : 5;
        cx<R> tmp[RAD];
#pragma unroll
        for (int r = 0; r < RAD; r++) tmp[r] = a[base + STRIDE * r];
#pragma unroll
        for (int r = 0; r < RAD; r++) {
            int rv = 0;
#pragma unroll
            for (int b = 0; b < LG; b++)
                if (r & (1 << b)) rv |= 1 << (LG - 1 - b);
            a[base + STRIDE * r] = tmp[rv];
        }
    }
}

template <int LOGN, int LOGE>
struct FftShape {
    static constexpr int N = 1 << LOGN;
    static constexpr int E = 1 << LOGE;
    static constexpr int T = N / E;
    static constexpr int NFULL = LOGN / LOGE;       // full radix-E passes
    static constexpr int REM = LOGN % LOGE;         // bits of the last pass
    static constexpr int NPASS = NFULL + (REM > 0 ? 1 : 0);
};

// Twiddle factors W_N^e = exp(-2 pi i e / N), e in [0, N), from a two-level
// table in shared memory: W^e = hi[e >> 6] * lo[e & 63] with both levels
// copied from the correctly rounded full table (product error ~2 ulp).
template <typename R, int LOGN>
struct Twiddles {
    static constexpr int N = 1 << LOGN;
    static constexpr int NLO = N < 64 ? N : 64;
    static constexpr int NHI = N / NLO;
    static constexpr int SIZE = NLO + (NHI > 1 ? NHI : 0);  // entries in smem
    const cx<R>* lo;
    const cx<R>* hi;
    __device__ __forceinline__ cx<R> operator()(int e) const {
        if constexpr (NHI == 1) return lo[e];
        else return cmul(hi[e >> 6], lo[e & 63]);
    }
    // fill from the full global table (all threads of the block; no sync)
    __device__ static void fill(cx<R>* dst, const cx<R>* __restrict__ full) {
        for (int i = threadIdx.x; i < SIZE; i += blockDim.x)
            dst[i] = i < NLO ? full[i] : full[(i - NLO) * NLO];
    }
    __device__ static Twiddles at(const cx<R>* base) {
        Twiddles t;
        t.lo = base;
        t.hi = base + NLO;
        return t;
    }
};

// The smem exchange moves whole complex values through one padded buffer,
// or -- when that buffer would not fit in shared memory (FP64 at 2^14
// points) -- the real and the imaginary parts in two rounds through a buffer
// of half the size.
template <typename R, int LOGN>
struct SmemPlan {
    static constexpr bool SPLIT = sizeof(R) * 2 * (size_t)padded_len(1 << LOGN) > 200 * 1024;
    static constexpr size_t BYTES =
        (SPLIT ? sizeof(R) : 2 * sizeof(R)) * (size_t)padded_len(1 << LOGN);
};

// Twiddles and radix-RP DFTs of one Stockham pass with stride ns (the product
// of the previous radices) on the E values of this thread.  The first pass
// (ns = 1) has no twiddles.
template <typename R, int LOGN, int LOGE, int RP, bool FIRST>
__device__ __forceinline__ void pass_compute(cx<R> (&v)[1 << LOGE], const Twiddles<R, LOGN>& tw,
                                             const int ns) {
    using S = FftShape<LOGN, LOGE>;
    constexpr int E = S::E, T = S::T, N = S::N;
    constexpr int BPT = E / RP;  // butterflies per thread
    const int t = threadIdx.x;
    const int tws = N / (ns * RP);
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        if constexpr (!FIRST) {
            const int m = (t + T * q) & (ns - 1);
            if constexpr (sizeof(R) == 8) {
                // FP64: powers of one table twiddle (rounding stays ~1e-15)
                const cx<R> w1 = tw(m * tws);
                cx<R> w = w1;
#pragma unroll
                for (int r = 1; r < RP; r++) {
                    v[q + BPT * r] = cmul(v[q + BPT * r], w);
                    if (r + 1 < RP) w = cmul(w, w1);
                }
            } else {
                // FP32: every twiddle from the correctly rounded table
#pragma unroll
                for (int r = 1; r < RP; r++) v[q + BPT * r] = cmul(v[q + BPT * r], tw(m * r * tws));
            }
        }
        dft_inreg<RP, false, BPT>(v, q);
    }
}

// Stockham reordering between passes: the outputs of a radix-RP pass with
// stride ns go to positions (j - m) RP + m + r ns; the next pass reads
// positions t + T s.  All threads of the block call it.
template <typename R, int LOGN, int LOGE, int RP>
__device__ __forceinline__ void pass_exchange(cx<R> (&v)[1 << LOGE], void* __restrict__ smv,
                                              const int ns) {
    using S = FftShape<LOGN, LOGE>;
    constexpr int E = S::E, T = S::T;
    constexpr int BPT = E / RP;
    const int t = threadIdx.x;
    if constexpr (!SmemPlan<R, LOGN>::SPLIT) {
        cx<R>* sm = (cx<R>*)smv;
#pragma unroll
        for (int q = 0; q < BPT; q++) {
            const int j = t + T * q, m = j & (ns - 1), base = (j - m) * RP + m;
#pragma unroll
            for (int r = 0; r < RP; r++) sm[pad(base + r * ns)] = v[q + BPT * r];
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = sm[pad(t + T * s)];
        __syncthreads();
    } else {
        R* sm = (R*)smv;
#pragma unroll
        for (int part = 0; part < 2; part++) {
#pragma unroll
            for (int q = 0; q < BPT; q++) {
                const int j = t + T * q, m = j & (ns - 1), base = (j - m) * RP + m;
#pragma unroll
                for (int r = 0; r < RP; r++)
                    sm[pad(base + r * ns)] = part ? v[q + BPT * r].im : v[q + BPT * r].re;
            }
            __syncthreads();
#pragma unroll
            for (int s = 0; s < E; s++) {
                if (part) v[s].im = sm[pad(t + T * s)];
                else v[s].re = sm[pad(t + T * s)];
            }
            __syncthreads();
        }
    }
}

// out[s] = value at position (N - (t + T s)) mod N of the field held in v
// (the k <-> -k pairing of two packed real spectra)
template <typename R, int LOGN, int LOGE>
__device__ __forceinline__ void gather_negated(const cx<R> (&v)[1 << LOGE], cx<R> (&out)[1 << LOGE],
                                               void* __restrict__ smv) {
    using S = FftShape<LOGN, LOGE>;
    constexpr int E = S::E, T = S::T, N = S::N;
    const int t = threadIdx.x;
    if constexpr (!SmemPlan<R, LOGN>::SPLIT) {
        cx<R>* sm = (cx<R>*)smv;
#pragma unroll
        for (int s = 0; s < E; s++) sm[pad(t + T * s)] = v[s];
        __syncthreads();
#pragma unroll
        for (int s = 0; s < E; s++) out[s] = sm[pad((N - (t + T * s)) & (N - 1))];
        __syncthreads();
    } else {
        R* sm = (R*)smv;
#pragma unroll
        for (int part = 0; part < 2; part++) {
#pragma unroll
            for (int s = 0; s < E; s++) sm[pad(t + T * s)] = part ? v[s].im : v[s].re;
            __syncthreads();
#pragma unroll
            for (int s = 0; s < E; s++) {
                const R x = sm[pad((N - (t + T * s)) & (N - 1))];
                if (part) out[s].im = x;
                else out[s].re = x;
            }
            __syncthreads();
        }
    }
}

// Split the spectrum X of two packed real sequences p + i q and apply
// v <- H P̂ + i conj(H) Q̂ in place, using X[k] and conj(X[-k]) read from
// shared memory one bin at a time (no second register array):
//   P̂ = (X[k] + conj(X[-k]))/2,  i Q̂ = (X[k] - conj(X[-k]))/2.
// H(k) returns the kernel at bin k.  All threads of the block call it.
template <typename R, int LOGN, int LOGE, class HF>
__device__ __forceinline__ void split_pair_apply(cx<R> (&v)[1 << LOGE], void* __restrict__ smv,
                                                 HF&& H) {
    using S = FftShape<LOGN, LOGE>;
    constexpr int E = S::E, T = S::T, N = S::N;
    const int t = threadIdx.x;
    if constexpr (!SmemPlan<R, LOGN>::SPLIT) {
        cx<R>* sm = (cx<R>*)smv;
#pragma unroll
        for (int s = 0; s < E; s++) sm[pad(t + T * s)] = v[s];
        __syncthreads();
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int b = t + T * s;
            const cx<R> zm = conjc(sm[pad((N - b) & (N - 1))]);
            const cx<R> h = H(b);
            const cx<R> a = scale(v[s] + zm, R(0.5));
            const cx<R> c = scale(v[s] - zm, R(0.5));
            v[s] = cmul(a, h) + cmulc(c, h);
        }
        __syncthreads();
    } else {
        // real and imaginary parts in two rounds through a half-size buffer
        R* sm = (R*)smv;
        R xr[E];
#pragma unroll
        for (int s = 0; s < E; s++) sm[pad(t + T * s)] = v[s].re;
        __syncthreads();
#pragma unroll
        for (int s = 0; s < E; s++) xr[s] = sm[pad((N - (t + T * s)) & (N - 1))];
        __syncthreads();
#pragma unroll
        for (int s = 0; s < E; s++) sm[pad(t + T * s)] = v[s].im;
        __syncthreads();
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int b = t + T * s;
            const cx<R> zm = mk(xr[s], -sm[pad((N - b) & (N - 1))]);
            const cx<R> h = H(b);
            const cx<R> a = scale(v[s] + zm, R(0.5));
            const cx<R> c = scale(v[s] - zm, R(0.5));
            v[s] = cmul(a, h) + cmulc(c, h);
        }
        __syncthreads();
    }
}

// Block-wide unnormalised forward transform (exponent sign -1) of the N
// values held in v; all threads of the block call it.  The passes between
// the first and the last run as a runtime loop over one code body, so a
// kernel carries one copy of each pass type.
template <typename R, int LOGN, int LOGE>
__device__ __forceinline__ void block_fft(cx<R> (&v)[1 << LOGE], void* sm,
                                          const Twiddles<R, LOGN>& tw) {
    using S = FftShape<LOGN, LOGE>;
    constexpr int E = S::E;
    constexpr int RL = S::REM ? (1 << S::REM) : E;  // radix of the last pass
    if constexpr (S::NPASS == 1) {
        dft_inreg<E, false, 1>(v, 0);
    } else {
        pass_compute<R, LOGN, LOGE, E, true>(v, tw, 1);
        pass_exchange<R, LOGN, LOGE, E>(v, sm, 1);
        int ns = E;
#pragma unroll 1
        for (int p = 1; p < S::NPASS - 1; p++) {
            pass_compute<R, LOGN, LOGE, E, false>(v, tw, ns);
            pass_exchange<R, LOGN, LOGE, E>(v, sm, ns);
            ns *= E;
        }
        pass_compute<R, LOGN, LOGE, RL, false>(v, tw, ns);
    }
}

// unnormalised inverse (exponent sign +1) through the forward code path:
// F⁻¹(x)·N = conj(F(conj(x)))
template <typename R, int E>
__device__ __forceinline__ void conj_all(cx<R> (&v)[E]) {
#pragma unroll
    for (int s = 0; s < E; s++) v[s].im = -v[s].im;
}

}  // namespace fl
