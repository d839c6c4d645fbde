// fl_sm_inst.cuh -- instantiation helper for the single-mode stepper.
#pragma once
#include "fl_launch.h"
#include "fl_sm.cuh"

namespace fl {

template <typename R, int LOGN, int LOGE>
cudaError_t launch_sm(const LaunchArgs& a) {
    using S = FftShape<LOGN, LOGE>;
    auto kern = sm_advance_kernel<R, LOGN, LOGE>;
    const size_t smem = sizeof(cx<R>) * padded_len(S::N) + 32 * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<a.nactive, S::T, smem, a.stream>>>(static_cast<const SlotDesc<R>*>(a.desc), a.state,
                                              a.active, a.max_evals);
    return cudaGetLastError();
}

template <typename R, int LOGN, int LOGE>
cudaError_t launch_rhs(const RhsArgs& a) {
    using S = FftShape<LOGN, LOGE>;
    auto kern = sm_rhs_kernel<R, LOGN, LOGE>;
    const size_t smem = sizeof(cx<R>) * padded_len(S::N) + 32 * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<1, S::T, smem, a.stream>>>(static_cast<const SlotDesc<R>*>(a.desc), a.adjoint, a.z,
                                      a.in, a.ufwd, a.out);
    return cudaGetLastError();
}

}  // namespace fl

#define FL_SM_INSTANCE(R, LOGN, LOGE)                                           \
    namespace fl {                                                              \
    cudaError_t launch_sm_##R##_##LOGN(const LaunchArgs& a) {                   \
        return launch_sm<R, LOGN, LOGE>(a);                                     \
    }                                                                           \
    cudaError_t launch_rhs_##R##_##LOGN(const RhsArgs& a) {                     \
        return launch_rhs<R, LOGN, LOGE>(a);                                    \
    }                                                                           \
    }
