// fl_dispatch.cu -- table of the built single-mode stepper instances.
#include "fl_launch.h"

namespace fl {

#define DECL(R, LOGN)                                          \
    cudaError_t launch_sm_##R##_##LOGN(const LaunchArgs&);     \
    cudaError_t launch_rhs_##R##_##LOGN(const RhsArgs&);
DECL(float, 6) DECL(float, 7) DECL(float, 8) DECL(float, 9) DECL(float, 10) DECL(float, 11)
DECL(float, 12) DECL(float, 13) DECL(float, 14)
DECL(double, 6) DECL(double, 7) DECL(double, 8) DECL(double, 9) DECL(double, 10)
DECL(double, 11) DECL(double, 12) DECL(double, 13)
#undef DECL

LaunchFn sm_launcher(int fp64, int logn) {
    static const LaunchFn f32[15] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                     launch_sm_float_6, launch_sm_float_7, launch_sm_float_8,
                                     launch_sm_float_9, launch_sm_float_10, launch_sm_float_11,
                                     launch_sm_float_12, launch_sm_float_13, launch_sm_float_14};
    static const LaunchFn f64[15] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                     launch_sm_double_6, launch_sm_double_7, launch_sm_double_8,
                                     launch_sm_double_9, launch_sm_double_10, launch_sm_double_11,
                                     launch_sm_double_12, launch_sm_double_13, nullptr};
    if (logn < 0 || logn > 14) return nullptr;
    return fp64 ? f64[logn] : f32[logn];
}

RhsFn rhs_launcher(int fp64, int logn) {
    static const RhsFn f32[15] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                  launch_rhs_float_6, launch_rhs_float_7, launch_rhs_float_8,
                                  launch_rhs_float_9, launch_rhs_float_10, launch_rhs_float_11,
                                  launch_rhs_float_12, launch_rhs_float_13, launch_rhs_float_14};
    static const RhsFn f64[15] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                  launch_rhs_double_6, launch_rhs_double_7, launch_rhs_double_8,
                                  launch_rhs_double_9, launch_rhs_double_10, launch_rhs_double_11,
                                  launch_rhs_double_12, launch_rhs_double_13, nullptr};
    if (logn < 0 || logn > 14) return nullptr;
    return fp64 ? f64[logn] : f32[logn];
}

int sm_threads(int fp64, int logn) {
    if (!sm_launcher(fp64, logn)) return 0;
    const int loge = logn <= 8 ? logn - 5 : (logn == 14 ? 5 : 4);
    return 1 << (logn - loge);
}

}  // namespace fl
