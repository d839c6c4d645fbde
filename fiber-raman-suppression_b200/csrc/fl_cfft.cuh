// fl_cfft.cuh -- Stockham FFT spread over a thread-block cluster of C CTAs.
//
// Used where one CTA cannot hold a transform (Nt = 2^15): the N values are
// held E per thread by the C*T threads of the cluster, global thread
// g = rank*T + tid owning positions g + C*T*s, exactly as block_fft does for
// one CTA.  The exchange buffer between passes is distributed: position p
// lives in the shared memory of CTA p / (N/C) at local index p mod (N/C), and
// each thread writes its pass outputs into the owning CTA's shared memory
// (distributed shared memory, st through a mapped generic address) and reads
// its next inputs the same way, with a cluster barrier (release/acquire) after
// each half of the exchange.  No TMA and no multicast are involved.
#pragma once
#include <cooperative_groups.h>

#include "fl_fft.cuh"

namespace fl {

template <int LOGN, int LOGE, int C>
struct ClusterShape {
    using S = FftShape<LOGN, LOGE>;
    static constexpr int N = S::N, E = S::E;
    static constexpr int TT = S::T;        // threads of the cluster
    static constexpr int T = TT / C;       // threads per CTA
    static constexpr int NL = N / C;       // positions held per CTA
    static_assert(TT % C == 0 && N % C == 0, "cluster split");
};

// bytes of one CTA's share of the exchange buffer (whole complex values)
template <typename R, int LOGN, int C>
constexpr size_t cluster_xbytes() {
    return 2 * sizeof(R) * (size_t)padded_len((1 << LOGN) / C);
}

__device__ __forceinline__ void cluster_sync_all() {
    cooperative_groups::this_cluster().sync();
}

// twiddles and radix-RP DFTs of one pass (pass_compute with the cluster's
// global thread index)
template <typename R, int LOGN, int LOGE, int C, int RP, bool FIRST>
__device__ __forceinline__ void cpass_compute(cx<R> (&v)[1 << LOGE], const Twiddles<R, LOGN>& tw,
                                              const int ns, const int g) {
    using CS = ClusterShape<LOGN, LOGE, C>;
    constexpr int E = CS::E, TT = CS::TT, N = CS::N;
    constexpr int BPT = E / RP;
    const int tws = N / (ns * RP);
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        if constexpr (!FIRST) {
            const int m = (g + TT * q) & (ns - 1);
            if constexpr (sizeof(R) == 8) {
                const cx<R> w1 = tw(m * tws);
                cx<R> w = w1;
#pragma unroll
                for (int r = 1; r < RP; r++) {
                    v[q + BPT * r] = cmul(v[q + BPT * r], w);
                    if (r + 1 < RP) w = cmul(w, w1);
                }
            } else {
#pragma unroll
                for (int r = 1; r < RP; r++) v[q + BPT * r] = cmul(v[q + BPT * r], tw(m * r * tws));
            }
        }
        dft_inreg<RP, false, BPT>(v, q);
    }
}

// Stockham reordering through the distributed buffer; sm is this CTA's share
template <typename R, int LOGN, int LOGE, int C, int RP>
__device__ __forceinline__ void cpass_exchange(cx<R> (&v)[1 << LOGE], cx<R>* __restrict__ sm,
                                               const int ns, const int g) {
    using CS = ClusterShape<LOGN, LOGE, C>;
    constexpr int E = CS::E, TT = CS::TT, NL = CS::NL;
    constexpr int BPT = E / RP;
    auto cl = cooperative_groups::this_cluster();
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        const int j = g + TT * q, m = j & (ns - 1), base = (j - m) * RP + m;
#pragma unroll
        for (int r = 0; r < RP; r++) {
            const int p = base + r * ns;
            cx<R>* dst = cl.map_shared_rank(sm, p / NL);
            dst[pad(p % NL)] = v[q + BPT * r];
        }
    }
    cl.sync();
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int p = g + TT * s;
        const cx<R>* src = cl.map_shared_rank(sm, p / NL);
        v[s] = src[pad(p % NL)];
    }
    cl.sync();
}

// unnormalised forward transform (sign -1) of the N values the cluster holds
template <typename R, int LOGN, int LOGE, int C>
__device__ __forceinline__ void cluster_fft(cx<R> (&v)[1 << LOGE], cx<R>* sm,
                                            const Twiddles<R, LOGN>& tw, const int g) {
    using S = FftShape<LOGN, LOGE>;
    constexpr int E = S::E;
    constexpr int RL = S::REM ? (1 << S::REM) : E;
    static_assert(S::NPASS > 1, "cluster transforms have more than one pass");
    cpass_compute<R, LOGN, LOGE, C, E, true>(v, tw, 1, g);
    cpass_exchange<R, LOGN, LOGE, C, E>(v, sm, 1, g);
    int ns = E;
#pragma unroll 1
    for (int p = 1; p < S::NPASS - 1; p++) {
        cpass_compute<R, LOGN, LOGE, C, E, false>(v, tw, ns, g);
        cpass_exchange<R, LOGN, LOGE, C, E>(v, sm, ns, g);
        ns *= E;
    }
    cpass_compute<R, LOGN, LOGE, C, RL, false>(v, tw, ns, g);
}

}  // namespace fl
