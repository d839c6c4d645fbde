// fl_mm_inst.cuh -- instantiation helper of the multimode evaluation round.
#pragma once
#include "fl_mm.cuh"
#include "fl_mm_launch.h"

namespace fl {

template <typename R, int LOGN, int LOGE>
cudaError_t mm_launch_fft_kernels(const MmRound& a, int which) {
    using S = FftShape<LOGN, LOGE>;
    const size_t smem = mm_smem_bytes<R, LOGN>();
    void (*k)(const MmDesc*, const MmState*, const int*) =
        which == 0 ? mm_prologue_kernel<R, LOGN, LOGE>
                   : which == 1 ? mm_pairs_kernel<R, LOGN, LOGE> : mm_epilogue_kernel<R, LOGN, LOGE>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid(which == 1 ? 2 * ((a.NP + 1) / 2) : a.M, a.nactive);
    k<<<grid, S::T, smem, a.stream>>>(static_cast<const MmDesc*>(a.desc), a.state, a.active);
    return cudaGetLastError();
}

template <int LOGN, int LOGE>
cudaError_t mm_round(const MmRound& a) {
    cudaError_t e;
#define FL_TRY(x)                        \
    if ((e = (x)) != cudaSuccess) return e;
    if (!a.fp64) FL_TRY((mm_launch_fft_kernels<float, LOGN, LOGE>(a, 0)));
    FL_TRY((mm_launch_fft_kernels<double, LOGN, LOGE>(a, 0)));
    FL_TRY(mm_launch_contract(a, 1));
    if (!a.fp64) FL_TRY((mm_launch_fft_kernels<float, LOGN, LOGE>(a, 1)));
    FL_TRY((mm_launch_fft_kernels<double, LOGN, LOGE>(a, 1)));
    FL_TRY(mm_launch_contract(a, 0));
    FL_TRY(mm_launch_contract(a, 2));
    if (!a.fp64) FL_TRY((mm_launch_fft_kernels<float, LOGN, LOGE>(a, 2)));
    FL_TRY((mm_launch_fft_kernels<double, LOGN, LOGE>(a, 2)));
    if (a.control) FL_TRY(mm_launch_control(a, 1));
#undef FL_TRY
    return cudaSuccess;
}

}  // namespace fl

#define FL_MM_INSTANCE(LOGN, LOGE)                                                   \
    namespace fl {                                                                   \
    cudaError_t mm_round_##LOGN(const MmRound& a) { return mm_round<LOGN, LOGE>(a); } \
    }
