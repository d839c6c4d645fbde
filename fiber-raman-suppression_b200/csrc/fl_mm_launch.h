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
    // slots with and without a low-rank form (rank > 0) may be in the batch:
    // the Z kernel serves the first, the Im X kernel the second; a kind known
    // to be absent is not launched
    int lowrank_some = 1, fullrank_some = 1;
    // a side stream (with two events) on which a stage's FP64 kernels run
    // beside its FP32 ones: they serve different slots or write different
    // buffers (nullptr: one stream)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int* ndone;            // control: count of finished slots (nullable)
    cudaStream_t stream;
};

using MmRoundFn = cudaError_t (*)(const MmRound&);

// Evidence reductions over saved spectra (fl_evidence.cuh).  Values per save
// position: [Σ tpow, max tpow, temporal edge sum, Σ spow, spectral edge sum,
// Σ |u|²/|ss|, then the M per-mode Σ_t |fft(u_m)|²], tpow and spow the
// mode-summed temporal and spectral power.
constexpr int kEvFixed = 6;
struct EvidenceArgs {
    const void* tw;          // FP64 twiddles exp(-2 pi i k / Nt)
    const double* ss;        // FP64 fftshift(ωs/ω0) (|ωs| = |ss| ω0)
    const double* spectra;   // nsave x M x Nt complex doubles, lab frame
    int nsave, M, N;
    double* out;             // nsave x (kEvFixed + M), device
    cudaStream_t stream;
};
using EvidenceFn = cudaError_t (*)(const EvidenceArgs&);
// evidence launcher for Nt = 2^logn (nullptr when not built)
EvidenceFn mm_evidence_launcher(int logn);

// evaluation round for Nt = 2^logn (nullptr when not built)
MmRoundFn mm_round_launcher(int logn);
// the grid-size-independent kernels (common translation unit)
cudaError_t mm_launch_contract(const MmRound& a, int which);  // 0 fwd, 1 Im X, 2 adjoint, 3 Z
cudaError_t mm_launch_control(const MmRound& a, int consume);
bool mm_supported_modes(int M);
// CTAs (one cluster) per transform at Nt = 2^logn
int mm_cluster_ctas(int logn);

}  // namespace fl
