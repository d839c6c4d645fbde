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

// returns nullptr when (precision, log2 Nt) is not built
LaunchFn sm_launcher(int fp64, int logn);
// threads per CTA of a built launcher (0 when not built)
int sm_threads(int fp64, int logn);

}  // namespace fl
