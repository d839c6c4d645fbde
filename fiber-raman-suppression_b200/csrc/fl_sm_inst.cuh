// fl_sm_inst.cuh -- instantiation helper for the single-mode stepper.
#pragma once
#include "fl_launch.h"
#include "fl_sm.cuh"

namespace fl {

template <typename RF, typename RA, int LOGN, int LOGE>
cudaError_t launch_sm(const LaunchArgs& a) {
    using S = FftShape<LOGN, LOGE>;
    auto kern = sm_advance_kernel<RF, RA, LOGN, LOGE>;
    const size_t smem = smem_bytes<RA, LOGN>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<a.nactive, S::T, smem, a.stream>>>(static_cast<const SlotDesc*>(a.desc), a.state,
                                              a.active, a.max_evals);
    return cudaGetLastError();
}

template <typename RF, typename RA, int LOGN, int LOGE>
cudaError_t launch_rhs(const RhsArgs& a) {
    using S = FftShape<LOGN, LOGE>;
    auto kern = sm_rhs_kernel<RF, RA, LOGN, LOGE>;
    const size_t smem = smem_bytes<RA, LOGN>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<1, S::T, smem, a.stream>>>(static_cast<const SlotDesc*>(a.desc), a.adjoint, a.z,
                                      a.in, a.ufwd, a.out);
    return cudaGetLastError();
}

}  // namespace fl

// NAME is the forward precision (float: FP32 forward with FP64 adjoint;
// double: FP64 throughout)
#define FL_SM_INSTANCE(NAME, RF, RA, LOGN, LOGE)                               \
    namespace fl {                                                              \
    cudaError_t launch_sm_##NAME##_##LOGN(const LaunchArgs& a) {                \
        return launch_sm<RF, RA, LOGN, LOGE>(a);                                \
    }                                                                           \
    cudaError_t launch_rhs_##NAME##_##LOGN(const RhsArgs& a) {                  \
        return launch_rhs<RF, RA, LOGN, LOGE>(a);                               \
    }                                                                           \
    }
