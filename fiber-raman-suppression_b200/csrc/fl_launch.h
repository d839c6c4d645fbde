// fl_launch.h -- launchers of the single-mode stepper, one per built grid size
// and precision; each is compiled in its own translation unit.
#pragma once
#include <cuda_runtime.h>

#include "fl_types.h"

namespace fl {

struct LaunchArgs {
    const void* desc;      // SlotDesc<R>[]
    SlotState* state;      // SlotState[]
    const int* active;     // slot indices, one CTA each
    int nactive;
    int max_evals;         // RHS evaluations per slot in this launch
    cudaStream_t stream;
};

using LaunchFn = cudaError_t (*)(const LaunchArgs&);

struct RhsArgs {
    const void* desc;      // one SlotDesc<R> (tables and scratch)
    int adjoint;
    double z;
    const double* in;      // N complex doubles: ũ or λ̃
    const double* ufwd;    // N complex doubles: forward field (adjoint)
    double* out;           // N complex doubles
    cudaStream_t stream;
};
using RhsFn = cudaError_t (*)(const RhsArgs&);
RhsFn rhs_launcher(int fp64, int logn);

// returns nullptr when (precision, log2 Nt) is not built
LaunchFn sm_launcher(int fp64, int logn);
// threads per CTA of a built launcher (0 when not built)
int sm_threads(int fp64, int logn);

// pump-gain forward solve of one single-mode problem (FP32 right-hand side,
// FP64 state and error norm), run to completion in one launch; false / an
// error when log2 Nt is not built (2^6..2^13)
bool gain_built(int logn);
cudaError_t launch_gain(int logn, const GainDesc* desc, GainOut* out, cudaStream_t stream);

}  // namespace fl
