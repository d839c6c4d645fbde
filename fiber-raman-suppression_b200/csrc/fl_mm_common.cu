// fl_mm_common.cu -- grid-size-independent multimode kernels (per-time
// contractions for each built mode count, the per-slot control kernel) and
// the table of evaluation rounds per grid size.
#include <algorithm>

#include "fl_mm.cuh"
#include "fl_mm_launch.h"
#include "fl_tc.cuh"

namespace fl {

#define DECL(LOGN) cudaError_t mm_round_##LOGN(const MmRound&);
DECL(6) DECL(7) DECL(8) DECL(9) DECL(10) DECL(11) DECL(12) DECL(13) DECL(14) DECL(15)
#undef DECL

MmRoundFn mm_round_launcher(int logn) {
    static const MmRoundFn f[16] = {nullptr,     nullptr,     nullptr,     nullptr,    nullptr,
                                    nullptr,     mm_round_6,  mm_round_7,  mm_round_8, mm_round_9,
                                    mm_round_10, mm_round_11, mm_round_12, mm_round_13,
                                    mm_round_14, mm_round_15};
    if (logn < 0 || logn > 15) return nullptr;
    return f[logn];
}

#define DECL_EV(LOGN) cudaError_t mm_evidence_##LOGN(const EvidenceArgs&);
DECL_EV(6) DECL_EV(7) DECL_EV(8) DECL_EV(9) DECL_EV(10) DECL_EV(11) DECL_EV(12) DECL_EV(13)
DECL_EV(14) DECL_EV(15)
#undef DECL_EV

EvidenceFn mm_evidence_launcher(int logn) {
    static const EvidenceFn f[16] = {nullptr,        nullptr,        nullptr,        nullptr,
                                     nullptr,        nullptr,        mm_evidence_6,  mm_evidence_7,
                                     mm_evidence_8,  mm_evidence_9,  mm_evidence_10, mm_evidence_11,
                                     mm_evidence_12, mm_evidence_13, mm_evidence_14, mm_evidence_15};
    if (logn < 0 || logn > 15) return nullptr;
    return f[logn];
}

int mm_cluster_ctas(int logn) { return logn == 15 ? 4 : 1; }

bool mm_supported_modes(int M) { return M >= 2 && M <= 10; }

__global__ void __launch_bounds__(kMmCtl)
    mm_control_kernel(const MmDesc* __restrict__ descs, MmState* __restrict__ states,
                      const int* __restrict__ active, int consume, int* __restrict__ ndone) {
    __shared__ double red[32];
    const int slot = active[blockIdx.x];
    const MmDesc& d = descs[slot];
    MmState st = states[slot];
    MmCtl c{d, st, red, (size_t)d.N * d.M, d.N};
    if (consume && mm_rhs_phase(st.phase) && st.phase != PH_EVAL_FWD && st.phase != PH_EVAL_ADJ)
        c.consume();
    __syncthreads();
    c.advance();
#ifdef FL_CHECKED
    // the indices the next evaluation's kernels will use (checked build)
    if (st.phase != PH_DONE && !state_in_bounds(d, st)) {
        st.status = ST_CHECK;
        st.phase = PH_DONE;
    }
#endif
    __syncthreads();
    if (threadIdx.x == 0) {
        states[slot] = st;
        if (ndone && st.phase == PH_DONE) atomicAdd(ndone, 1);
    }
}


// The FP32 forward contraction on the tensor cores (M >= 6, Nt a multiple
// of 128): CTAs loop over a slot's 128-point tiles.
template <int M>
__global__ void __launch_bounds__(kTcRows)
    mm_contract_tc_kernel(const MmDesc* __restrict__ descs, const MmState* __restrict__ states,
                          const int* __restrict__ active) {
    extern __shared__ __align__(16) unsigned char tc_smem[];
    const int slot = active[blockIdx.y];
    const MmDesc& d = descs[slot];
    if (d.M != M) return;
    const MmState st = states[slot];
    if (!mm_takes<float>(d, st) || mm_adjoint_phase(st.phase)) return;
    mm_contract_fwd_tc<M>(d, blockIdx.x, gridDim.x, tc_smem);
}

// The adjoint assembly of FP32-forward batches with the forward-field
// contractions on the tensor cores (M >= 6, Nt a multiple of 128): one
// 128-point tile per CTA.
template <int M>
__global__ void __launch_bounds__(kTcRows, 2)
    mm_contract_adj_tc_kernel(const MmDesc* __restrict__ descs, const MmState* __restrict__ states,
                              const int* __restrict__ active) {
    extern __shared__ __align__(16) unsigned char tc_smem[];
    const int slot = active[blockIdx.y];
    const MmDesc& d = descs[slot];
    if (d.M != M || !d.adj_mixed) return;
    const MmState st = states[slot];
    if (!mm_takes<double>(d, st) || !mm_adjoint_phase(st.phase)) return;
    mm_contract_adj_tc<M>(d, blockIdx.x, tc_smem);
}

// The adjoint's Im X contraction of FP32-forward batches on the tensor
// cores (M >= 6, Nt a multiple of 128): one 128-point tile per CTA.
template <int M>
__global__ void __launch_bounds__(kTcRows, 2)
    mm_imx_tc_kernel(const MmDesc* __restrict__ descs, const MmState* __restrict__ states,
                     const int* __restrict__ active) {
    extern __shared__ __align__(16) unsigned char tc_smem[];
    const int slot = active[blockIdx.y];
    const MmDesc& d = descs[slot];
    // (with a low-rank form the Z kernel reduces Y to the rank instead)
    if (d.M != M || !d.adj_mixed || d.rank > 0) return;
    const MmState st = states[slot];
    if (!mm_takes<double>(d, st) || !mm_adjoint_phase(st.phase)) return;
    mm_imx_tc<M>(d, blockIdx.x, tc_smem);
}

// The low-rank form's Z reduction (rank > 0): every RHS evaluation of an
// FP32 batch (forward, and the mixed adjoint's forward field).
template <int M>
__global__ void __launch_bounds__(kTcRows, 2)
    mm_z_tc_kernel(const MmDesc* __restrict__ descs, const MmState* __restrict__ states,
                   const int* __restrict__ active) {
    extern __shared__ __align__(16) unsigned char tc_smem[];
    const int slot = active[blockIdx.y];
    const MmDesc& d = descs[slot];
    if (d.M != M || d.rank <= 0 || d.fp64) return;
    const MmState st = states[slot];
    if (!mm_rhs_phase(st.phase)) return;
    mm_z_tc<M>(d, blockIdx.x, tc_smem, mm_adjoint_phase(st.phase));
}

namespace {

template <int M>
cudaError_t z_tc(const MmRound& a) {
    const size_t smem = TcShape<M>::SMEM;
    cudaError_t e = cudaFuncSetAttribute(mm_z_tc_kernel<M>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid(a.N / kTcRows, a.nactive);
    mm_z_tc_kernel<M><<<grid, kTcRows, smem, a.stream>>>(static_cast<const MmDesc*>(a.desc),
                                                        a.state, a.active);
    return cudaGetLastError();
}

template <int M>
cudaError_t imx_tc(const MmRound& a) {
    const size_t smem = TcSymShape<M>::SMEM;
    cudaError_t e = cudaFuncSetAttribute(mm_imx_tc_kernel<M>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid(a.N / kTcRows, a.nactive);
    mm_imx_tc_kernel<M><<<grid, kTcRows, smem, a.stream>>>(static_cast<const MmDesc*>(a.desc),
                                                          a.state, a.active);
    return cudaGetLastError();
}

template <int M>
cudaError_t contract_adj_tc(const MmRound& a) {
    const size_t smem = TcSymShape<M>::SMEM_LAUNCH;
    cudaError_t e = cudaFuncSetAttribute(mm_contract_adj_tc_kernel<M>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid(a.N / kTcRows, a.nactive);
    mm_contract_adj_tc_kernel<M><<<grid, kTcRows, smem, a.stream>>>(
        static_cast<const MmDesc*>(a.desc), a.state, a.active);
    return cudaGetLastError();
}

template <int M>
cudaError_t contract_tc(const MmRound& a) {
    const size_t smem = TcShape<M>::SMEM;
    cudaError_t e = cudaFuncSetAttribute(mm_contract_tc_kernel<M>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // one 128-point tile per CTA (many CTAs in flight hide each tile's
    // load -> MMA -> drain chain better than a persistent loop)
    const dim3 grid(a.N / kTcRows, a.nactive);
    mm_contract_tc_kernel<M><<<grid, kTcRows, smem, a.stream>>>(
        static_cast<const MmDesc*>(a.desc), a.state, a.active);
    return cudaGetLastError();
}

template <typename R, int M>
cudaError_t contract_m(const MmRound& a, int which) {
    // which = 3: the low-rank form's Z reduction (FP32 batches with M >= 6;
    // slots without a low-rank form skip it)
    if (which == 3) {
        if constexpr (M >= 6) {
            if (mm_adj_mixed(M, a.N, a.fp64) && a.lowrank_some) return z_tc<M>(a);
        }
        return cudaSuccess;
    }
    // FP32 forward with M >= 6 modes: tensor cores (3xTF32)
    if constexpr (sizeof(R) == 4 && M >= 6) {
        if (which == 0 && a.tensor_cores && a.N % kTcRows == 0) return contract_tc<M>(a);
    }
    // mixed-precision adjoint (mm_adj_mixed): the assembly's forward-field
    // contractions and the Im X contraction on the tensor cores (3xTF32)
    if constexpr (sizeof(R) == 8 && M >= 6) {
        if (which == 2 && mm_adj_mixed(M, a.N, a.fp64)) return contract_adj_tc<M>(a);
        if (which == 1 && mm_adj_mixed(M, a.N, a.fp64))
            return a.fullrank_some ? imx_tc<M>(a) : cudaSuccess;
    }
    const int n = which == 2 ? a.N * M : a.N;
    const dim3 grid((n + kMmTB - 1) / kMmTB, a.nactive);
    mm_contract_kernel<R, M><<<grid, kMmTB, 0, a.stream>>>(static_cast<const MmDesc*>(a.desc),
                                                          a.state, a.active, which);
    return cudaGetLastError();
}

template <typename R>
cudaError_t contract_r(const MmRound& a, int which) {
    switch (a.M) {
        case 1: return contract_m<R, 1>(a, which);
        case 2: return contract_m<R, 2>(a, which);
        case 3: return contract_m<R, 3>(a, which);
        case 4: return contract_m<R, 4>(a, which);
        case 5: return contract_m<R, 5>(a, which);
        case 6: return contract_m<R, 6>(a, which);
        case 7: return contract_m<R, 7>(a, which);
        case 8: return contract_m<R, 8>(a, which);
        case 9: return contract_m<R, 9>(a, which);
        case 10: return contract_m<R, 10>(a, which);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t mm_launch_contract(const MmRound& a, int which) {
    // the forward contraction runs in the batch's forward precision; the
    // adjoint passes in FP64
    if (which == 0 && !a.fp64) return contract_r<float>(a, which);
    return contract_r<double>(a, which);
}

cudaError_t mm_launch_control(const MmRound& a, int consume) {
    mm_control_kernel<<<a.nactive, kMmCtl, 0, a.stream>>>(static_cast<const MmDesc*>(a.desc),
                                                          a.state, a.active, consume, a.ndone);
    return cudaGetLastError();
}

}  // namespace fl
