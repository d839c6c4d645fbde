// fl_evidence.cuh -- on-device FP64 evidence reductions over saved spectra.
//
// The reference's propagate evidence (src/fiberlab/propagation.jl:176-237:
// _edge_fraction, _photon_number, _field_metrics, _propagation_metrics)
// reduces each saved lab-frame spectrum u (M modes x Nt bins):
//   temporal field        fft(u) along time (unnormalised, sign -1)
//   mode energy [pJ]      Δt Σ_t |fft(u_m)|²
//   peak power [W]        max_t Σ_m |fft(u_m)(t)|²
//   edge fractions        power in the first and last max(1, floor(0.05 Nt))
//                         samples over the total, of the mode-summed temporal
//                         power and of the fftshift-ed spectral power
//   photon number         Δt Σ |u|² / fftshift(|ωs|)
// One transform group (a CTA, or a cluster at Nt = 2^15) per save position
// loops over the modes: each thread owns the same bins in every transform,
// so the mode sum of the temporal power stays in its registers.  The kernel
// returns the raw FP64 sums; the host scales them by Δt and 1/ω0 (grid
// constants the tables do not carry).  Sums run in a fixed order (block
// shuffle tree, then the cluster's ranks in order), so results are
// reproducible run to run.
#pragma once
#include "fl_mm.cuh"
#include "fl_mm_launch.h"

namespace fl {

// sum (or max) over the transform group: the CTA's block reduction, then,
// for a cluster, the ranks' values in rank order through rank 0's shared
// memory (xch holds one double per rank)
template <int T, int CL>
__device__ __forceinline__ double group_reduce(double v, bool is_max, double* red, double* xch,
                                               int rank) {
    const double b = is_max ? block_max<T>(v, red) : block_sum<T>(v, red);
    if constexpr (CL == 1) {
        return b;
    } else {
        auto cl = cooperative_groups::this_cluster();
        if (threadIdx.x == 0) *cl.map_shared_rank(xch + rank, 0) = b;
        cl.sync();
        const double* x0 = cl.map_shared_rank(xch, 0);
        double r = x0[0];
#pragma unroll
        for (int c = 1; c < CL; c++) r = is_max ? fmax(r, x0[c]) : r + x0[c];
        cl.sync();  // the slots are reused by the next reduction
        return r;
    }
}

template <int LOGN, int LOGE, int CL>
__global__ void __launch_bounds__(MmGroup<double, LOGN, LOGE, CL>::T, 1)
    evidence_kernel(const MmDesc tab, const double* __restrict__ spectra,
                    const double* __restrict__ ss, int M, double* __restrict__ out) {
    using G = MmGroup<double, LOGN, LOGE, CL>;
    constexpr int N = G::N, E = G::E, TT = G::TT, T = G::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int s = blockIdx.x / CL;
    G grp;
    grp.init(tab, smraw);
    double* xch = grp.red + 32;
    const int g = grp.g;
    const int k = max(1, (int)floor(0.05 * (double)N));  // _edge_fraction's edge width
    const double* base = spectra + (size_t)s * M * N * 2;
    double* o = out + (size_t)s * (kEvFixed + M);
    double tp[E];
#pragma unroll
    for (int e = 0; e < E; e++) tp[e] = 0.0;
    double sp_tot = 0.0, sp_edge = 0.0, photon = 0.0;
#pragma unroll 1
    for (int m = 0; m < M; m++) {
        cx<double> v[E];
#pragma unroll
        for (int e = 0; e < E; e++) {
            const int b = g + TT * e;
            v[e] = ld2(base + (size_t)m * N * 2, b);
            const double a = energy(v[e]);
            sp_tot += a;
            const int j = (b + N / 2) & (N - 1);  // position in fftshift order
            if (j < k || j >= N - k) sp_edge += a;
            photon += a / fabs(ss[b]);
        }
        grp.fft(v);
        double me = 0.0;
#pragma unroll
        for (int e = 0; e < E; e++) {
            const double t = energy(v[e]);
            tp[e] += t;
            me += t;
        }
        me = group_reduce<T, CL>(me, false, grp.red, xch, grp.rank);
        if (grp.rank == 0 && threadIdx.x == 0) o[kEvFixed + m] = me;
    }
    double t_tot = 0.0, t_max = 0.0, t_edge = 0.0;
#pragma unroll
    for (int e = 0; e < E; e++) {
        const int b = g + TT * e;
        t_tot += tp[e];
        t_max = fmax(t_max, tp[e]);
        if (b < k || b >= N - k) t_edge += tp[e];
    }
    t_tot = group_reduce<T, CL>(t_tot, false, grp.red, xch, grp.rank);
    t_max = group_reduce<T, CL>(t_max, true, grp.red, xch, grp.rank);
    t_edge = group_reduce<T, CL>(t_edge, false, grp.red, xch, grp.rank);
    sp_tot = group_reduce<T, CL>(sp_tot, false, grp.red, xch, grp.rank);
    sp_edge = group_reduce<T, CL>(sp_edge, false, grp.red, xch, grp.rank);
    photon = group_reduce<T, CL>(photon, false, grp.red, xch, grp.rank);
    if (grp.rank == 0 && threadIdx.x == 0) {
        o[0] = t_tot;
        o[1] = t_max;
        o[2] = t_edge;
        o[3] = sp_tot;
        o[4] = sp_edge;
        o[5] = photon;
    }
}

template <int LOGN, int LOGE, int CL>
cudaError_t launch_evidence(const EvidenceArgs& a) {
    using G = MmGroup<double, LOGN, LOGE, CL>;
    const size_t smem = G::SMEM + 64 * sizeof(double);  // + the cluster exchange slots
    auto k = evidence_kernel<LOGN, LOGE, CL>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    MmDesc tab{};
    tab.tw[1] = a.tw;
    tab.N = a.N;
    tab.M = a.M;
    if constexpr (CL == 1) {
        k<<<a.nsave, G::T, smem, a.stream>>>(tab, a.spectra, a.ss, a.M, a.out);
        return cudaGetLastError();
    } else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(a.nsave * CL);
        cfg.blockDim = dim3(G::T);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = a.stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = CL;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, k, tab, a.spectra, a.ss, a.M, a.out);
    }
}

}  // namespace fl
