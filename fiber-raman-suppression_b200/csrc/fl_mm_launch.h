// fl_mm_launch.h -- launchers of the multimode stepper: one evaluation round
// (prologue, Im X, pairs, contraction, epilogue, control) over the active
// slots, per built grid size.
#pragma once
#include <cuda_runtime.h>

#include "fl_types.h"

namespace fl {

struct MmRound {
    const void* desc;      // MmDesc[]
    MmState* state;        // MmState[]
    const int* active;     // slot indices
    int nactive;
    int M, NP, N;          // modes, pairs, points (same for every slot of the batch)
    int fp64;              // forward precision of the batch
    int control;           // run the control kernel after the evaluation
    int tensor_cores;      // FP32 forward contraction on tcgen05 when M >= 6
    int* ndone;            // control: count of finished slots (nullable)
    cudaStream_t stream;
};

using MmRoundFn = cudaError_t (*)(const MmRound&);

// evaluation round for Nt = 2^logn (nullptr when not built)
MmRoundFn mm_round_launcher(int logn);
// the grid-size-independent kernels (common translation unit)
cudaError_t mm_launch_contract(const MmRound& a, int which);  // 0 fwd, 1 Im X, 2 adjoint
cudaError_t mm_launch_control(const MmRound& a, int consume);
bool mm_supported_modes(int M);
// CTAs (one cluster) per transform at Nt = 2^logn
int mm_cluster_ctas(int logn);

}  // namespace fl
