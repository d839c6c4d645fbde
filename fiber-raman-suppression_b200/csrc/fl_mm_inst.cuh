// fl_mm_inst.cuh -- instantiation helper of the multimode evaluation round.
#pragma once
#include <nvtx3/nvToolsExt.h>

#include "fl_evidence.cuh"
#include "fl_mm.cuh"
#include "fl_mm_launch.h"

namespace fl {

// which: 0 prologue, 1 pairs, 2 epilogue; CL CTAs (one cluster) per transform
template <typename R, int LOGN, int LOGE, int CL>
cudaError_t mm_launch_fft_kernels(const MmRound& a, int which) {
    using G = MmGroup<R, LOGN, LOGE, CL>;
    const size_t smem = G::SMEM;
    void (*k)(const MmDesc*, const MmState*, const int*) =
        which == 0   ? mm_prologue_kernel<R, LOGN, LOGE, CL>
        : which == 1 ? mm_pairs_kernel<R, LOGN, LOGE, CL>
                     : mm_epilogue_kernel<R, LOGN, LOGE, CL>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int units = which == 1 ? 2 * ((a.NP + 1) / 2) : a.M;
    const dim3 grid(units * CL, a.nactive);
    if constexpr (CL == 1) {
        k<<<grid, G::T, smem, a.stream>>>(static_cast<const MmDesc*>(a.desc), a.state, a.active);
        return cudaGetLastError();
    } else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
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
        return cudaLaunchKernelEx(&cfg, k, static_cast<const MmDesc*>(a.desc),
                                  static_cast<const MmState*>(a.state), a.active);
    }
}

// one evaluation round; each stage's launches sit in a named NVTX range
// (host-side: under graph capture the ranges mark the capture)
template <int LOGN, int LOGE, int CL>
cudaError_t mm_round(const MmRound& a) {
    cudaError_t e;
#define FL_TRY(x)                        \
    if ((e = (x)) != cudaSuccess) {      \
        nvtxRangePop();                  \
        return e;                        \
    }
    // FP32 batches with a side stream: each stage's FP64 kernel runs on it,
    // beside the FP32 one (the two serve forward and adjoint slots, or write
    // the forward field's and λ's buffers), joined before the next stage
    const bool two = a.side != nullptr && !a.fp64;
    MmRound b = a;
    if (two) b.stream = a.side;
    auto fork = [&]() -> cudaError_t {
        if (!two) return cudaSuccess;
        cudaError_t x = cudaEventRecord(a.ev_fork, a.stream);
        return x == cudaSuccess ? cudaStreamWaitEvent(a.side, a.ev_fork, 0) : x;
    };
    auto join = [&]() -> cudaError_t {
        if (!two) return cudaSuccess;
        cudaError_t x = cudaEventRecord(a.ev_join, a.side);
        return x == cudaSuccess ? cudaStreamWaitEvent(a.stream, a.ev_join, 0) : x;
    };
    nvtxRangePushA("fl: mm prologue");
    FL_TRY(fork());
    if (!a.fp64) FL_TRY((mm_launch_fft_kernels<float, LOGN, LOGE, CL>(a, 0)));
    FL_TRY((mm_launch_fft_kernels<double, LOGN, LOGE, CL>(b, 0)));
    FL_TRY(join());
    nvtxRangePop();
    nvtxRangePushA("fl: mm Im X contraction");
    FL_TRY(mm_launch_contract(a, 1));
    nvtxRangePop();
    nvtxRangePushA("fl: mm low-rank reduction");
    FL_TRY(mm_launch_contract(a, 3));
    nvtxRangePop();
    nvtxRangePushA("fl: mm pairs");
    FL_TRY(fork());
    if (!a.fp64) FL_TRY((mm_launch_fft_kernels<float, LOGN, LOGE, CL>(a, 1)));
    FL_TRY((mm_launch_fft_kernels<double, LOGN, LOGE, CL>(b, 1)));
    FL_TRY(join());
    nvtxRangePop();
    nvtxRangePushA("fl: mm contraction");
    FL_TRY(fork());
    FL_TRY(mm_launch_contract(a, 0));
    FL_TRY(mm_launch_contract(b, 2));
    FL_TRY(join());
    nvtxRangePop();
    nvtxRangePushA("fl: mm epilogue");
    FL_TRY(fork());
    if (!a.fp64) FL_TRY((mm_launch_fft_kernels<float, LOGN, LOGE, CL>(a, 2)));
    FL_TRY((mm_launch_fft_kernels<double, LOGN, LOGE, CL>(b, 2)));
    FL_TRY(join());
    nvtxRangePop();
    if (a.control) {
        nvtxRangePushA("fl: mm control");
        FL_TRY(mm_launch_control(a, 1));
        nvtxRangePop();
    }
#undef FL_TRY
    return cudaSuccess;
}

}  // namespace fl

#define FL_MM_INSTANCE(LOGN, LOGE, CL)                                                     \
    namespace fl {                                                                         \
    cudaError_t mm_round_##LOGN(const MmRound& a) { return mm_round<LOGN, LOGE, CL>(a); } \
    cudaError_t mm_evidence_##LOGN(const EvidenceArgs& a) {                                \
        return launch_evidence<LOGN, LOGE, CL>(a);                                         \
    }                                                                                      \
    }
