// fl_tc.cuh -- the multimode stepper's per-time-point contractions on the
// 5th-generation tensor cores (tcgen05, sm_100a), for M >= 6 modes: the
// forward Kerr/Raman contraction (below), the adjoint's Im X reduction and
// assembly (mm_imx_tc, mm_contract_adj_tc) and the low-rank form's
// reductions (mm_z_tc).  In the low-rank form (rank > 0) the forward GEMM
// takes B = U and A = S̃ (K = the rank padded to 8) instead of G and S.
//
// Per time point t the forward contraction is δ_ij(t) = Σ_q G[ij][q] S_q(t)
// followed by η_i = Σ_j δ_ij u_j (simulate_disp_mmf.jl:38-53 with the Raman
// convolution folded into S).  Over a tile of 128 time points the first step
// is a GEMM D[t][ij] = Σ_q A[t][q] B[ij][q] with A = S (128 x NP) and B = G
// (M² x NP), both K-major: one tcgen05.mma of kind::tf32 per 8 pairs, the
// accumulator D (fp32, 128 lanes x M² columns) in tensor memory.  FP32
// accuracy comes from the 3xTF32 split: x = hi + lo with hi, lo exact TF32
// values, D = A_hi B_hi + A_hi B_lo + A_lo B_hi.
//
// Shared-memory operands use the canonical K-major layout without swizzle:
// core matrices of 8 rows x 16 bytes (8 x 4 TF32 values) stored as 128
// contiguous bytes; core matrices adjacent along K are LBO = 128 bytes apart
// and those adjacent along M/N are SBO = KP*32 bytes apart (KP = the pair
// count padded to 8, zeros beyond).  The k-th MMA (pairs 8k..8k+7) starts
// 256 bytes after the (k-1)-th.
//
// One elected thread issues the MMAs and commits them to an mbarrier; every
// thread waits on it with a bounded spin (on timeout the tile's outputs are
// set to NaN, which the error norm turns into FL_NONFINITE) and then reads
// its own row of D with tcgen05.ld.  Tensor memory is allocated per CTA
// (128 columns for the forward GEMM) and freed before the CTA exits on every
// path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fl_fft.cuh"
#include "fl_types.h"

namespace fl {

constexpr int kTcRows = 128;  // time points per tile = MMA M = threads per CTA

__host__ __device__ constexpr int tc_nn(int M) { return (M * M + 15) & ~15; }           // MMA N
__host__ __device__ constexpr int tc_kp(int M) { return (M * (M + 1) / 2 + 7) & ~7; }  // K padded to 8

template <int M>
struct TcShape {
    static constexpr int NP = M * (M + 1) / 2;
    static constexpr int KP = tc_kp(M);                 // whole MMAs of 8 pairs
    static constexpr int GP = mm_gp(M);                 // row stride of the G table
    static constexpr int NN = tc_nn(M);
    static constexpr int SBO = KP * 32;                 // bytes between 8-row groups
    static constexpr int A_BYTES = kTcRows * KP * 4;    // one of A_hi / A_lo
    static constexpr int B_BYTES = NN * KP * 4;         // one of B_hi / B_lo
    static constexpr int SMEM = 2 * A_BYTES + 2 * B_BYTES + 64 + 1024;  // + barrier, slack for alignment
    static_assert(NN <= 128, "accumulator columns");
    static_assert(SBO / 16 < (1 << 14), "SBO field");
};

// byte offset of element (row r, k) in a K-major no-swizzle tile
__host__ __device__ constexpr uint32_t tc_off_rt(int r, int k, int KP) {
    return (uint32_t)((r >> 3) * (KP * 32) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}
template <int KP>
__device__ __forceinline__ uint32_t tc_off(int r, int k) {
    return (uint32_t)((r >> 3) * (KP * 32) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

// TF32 round-to-nearest (the 10-bit mantissa value, low 13 bits zero)
__device__ __forceinline__ float tf32_rn(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// shared-memory matrix descriptor (K-major, no swizzle, sm_100 version 1)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    return d;                // base offset 0, LBO mode 0, layout SWIZZLE_NONE (0)
}

// instruction descriptor: D f32, A and B tf32, both K-major, shape 128 x N
__host__ __device__ constexpr uint32_t tc_idesc(int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// 3 x kp/8 MMAs (3xTF32) of one A tile against B (both kp pairs deep, K-major,
// split hi/lo) into the accumulator at tmem; n = the MMA's N (rows of B)
__device__ __forceinline__ void tc_issue3(uint32_t tmem, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi,
                                          uint32_t b_lo, int kp, int n) {
    const uint32_t idesc = tc_idesc(n);
    const uint32_t sbo = (uint32_t)kp * 32;
#pragma unroll 1
    for (int ks = 0; ks < kp / 8; ks++) {
        const uint32_t koff = (uint32_t)ks * 256;
        const uint64_t dah = tc_desc(a_hi + koff, 128, sbo);
        const uint64_t dal = tc_desc(a_lo + koff, 128, sbo);
        const uint64_t dbh = tc_desc(b_hi + koff, 128, sbo);
        const uint64_t dbl = tc_desc(b_lo + koff, 128, sbo);
        const uint32_t acc0 = ks > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(dah), "l"(dbh), "r"(idesc), "r"(acc0));
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(dah), "l"(dbl), "r"(idesc), "r"(1u));
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(dal), "l"(dbh), "r"(idesc), "r"(1u));
    }
}


// The forward contraction of the 128-point tiles t0 = tile*128, tile =
// first, first + step, ... < N/128 of one slot.  The B operand (the G table,
// split hi/lo) and the tensor memory are set up once per CTA; each tile
// refills A, issues its MMAs and waits on the barrier's next phase.
template <int M>
__device__ void mm_contract_fwd_tc(const MmDesc& d, int first, int step, unsigned char* smem) {
    using TS = TcShape<M>;
    constexpr int NN = TS::NN;
    const int N = d.N, ntiles = N / kTcRows;
    const int tid = threadIdx.x, warp = tid >> 5;
    // K of the GEMM: the pairs, or in the low-rank form the rank (A = S̃_k,
    // B = U); both padded to whole MMAs of 8
    const int nk = d.rank > 0 ? d.rank : TS::NP;
    const int kp = (nk + 7) & ~7;
    // 1024-byte aligned operand area (laid out for this K; sized for the largest)
    unsigned char* base =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem) + 1023) & ~uintptr_t(1023));
    const uint32_t a_bytes = (uint32_t)kTcRows * kp * 4, b_bytes = (uint32_t)NN * kp * 4;
    unsigned char* Ahi = base;
    unsigned char* Alo = Ahi + a_bytes;
    unsigned char* Bhi = Alo + a_bytes;
    unsigned char* Blo = Bhi + b_bytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(base + 2 * TS::A_BYTES + 2 * TS::B_BYTES);  // MMA completion
    uint64_t* bbar = mbar + 1;                                         // B-image arrival
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2);
    uint32_t* bfail = tmem_slot + 1;                                   // B copy timed out

    // ---- tensor memory and barrier
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(128));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // ---- B = G rows (ij) x pairs, split hi/lo: the image prepared once per
    // problem in exactly this shared-memory layout (B_hi then B_lo), brought in
    // by the TMA engine as bulk copies (16-byte aligned, sizes multiples of 16)
    // completing on bbar, while the threads build the first A tile
    const uint32_t kBBytes = 2 * b_bytes, kBChunk = 16384;  // a multiple of 16 (kp of 8)
    if (tid == 0) {
        *bfail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                         smem_u32(bbar)),
                     "r"(kBBytes)
                     : "memory");
        const char* src = reinterpret_cast<const char*>(d.rank > 0 ? d.Utc : d.Gtc);
        for (uint32_t off = 0; off < kBBytes; off += kBChunk) {
            const uint32_t n = kBBytes - off < kBChunk ? kBBytes - off : kBChunk;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
                "[%3];" ::"r"(smem_u32(Bhi) + off),
                "l"(src + off), "r"(n), "r"(smem_u32(bbar))
                : "memory");
        }
    }
    bool b_waited = false;  // thread 0: the B image has been waited for

    const float* sq = static_cast<const float*>(d.sq);
    const cx<float>* ut = static_cast<const cx<float>*>(d.ut);
    cx<float>* eta = static_cast<cx<float>*>(d.eta);
    uint32_t phase = 0;
    bool ok = true;
    int mma_pending = -1;  // parity of a commit whose arrival a timed-out wait did not see
    for (int tile = first; tile < ntiles; tile += step) {
        const int t = tile * kTcRows + tid;
        if (!ok) {  // an earlier tile timed out: no more MMAs from this CTA
#pragma unroll
            for (int i = 0; i < M; i++) eta[(size_t)i * N + t] = mk(__int_as_float(0x7fc00000), 0.f);
            continue;
        }
        // ---- A = this tile's S (or S̃), split hi/lo: four per 16-byte store
#pragma unroll 2
        for (int k = 0; k < kp; k += 4) {
            float4 hi, lo;
            float* h = &hi.x;
            float* l = &lo.x;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const float s = k + c < nk ? sq[(size_t)(k + c) * N + t] : 0.f;
                h[c] = tf32_rn(s);
                l[c] = tf32_rn(s - h[c]);
            }
            *reinterpret_cast<float4*>(Ahi + tc_off_rt(tid, k, kp)) = hi;
            *reinterpret_cast<float4*>(Alo + tc_off_rt(tid, k, kp)) = lo;
        }
        // generic-proxy shared stores -> visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tmem = *tmem_slot;

        // ---- 3 x KP/8 MMAs from one thread, committed to the barrier (after a
        // bounded wait for the B image on the first tile; if it does not land
        // the tile is flagged and no MMA is issued)
        if (tid == 0 && !b_waited) {
            uint32_t got = 0;
            for (long it = 0; it < (1L << 26) && !got; it++) {
                asm volatile(
                    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}\n"
                    : "=r"(got)
                    : "r"(smem_u32(bbar))
                    : "memory");
            }
            b_waited = true;
            if (!got) *bfail = 1;
        }
        if (tid == 0 && !*bfail)
            tc_issue3(tmem, smem_u32(Ahi), smem_u32(Alo), smem_u32(Bhi), smem_u32(Blo), kp, NN);
        if (tid == 0)  // arrives once the MMAs above (if any) have completed
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(mbar))
                : "memory");

        // ---- bounded wait for this tile's MMAs (the barrier's current phase)
        uint32_t done = 0;
        for (long it = 0; it < (1L << 26) && !done; it++) {
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done)
                : "r"(smem_u32(mbar)), "r"(phase)
                : "memory");
        }
        if (!done && mma_pending < 0) mma_pending = (int)phase;
        phase ^= 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        ok = ok && done;

        // ---- this thread's row of D: columns ij = i*M + j
        float dv[NN];
        if (ok) {
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
            for (int c = 0; c < NN; c += 16) {
                uint32_t r[16];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, "
                    "%9, %10, %11, %12, %13, %14, %15}, [%16];\n"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                      "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                      "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                    : "r"(taddr + (uint32_t)c));
#pragma unroll
                for (int q = 0; q < 16; q++) dv[c + q] = __uint_as_float(r[q]);
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        }
        // the next tile's MMAs overwrite the accumulator and A: all reads done
        // first.  The barrier also makes ok block-uniform (a wait that gave up
        // in any thread stops the CTA's MMAs), so every thread takes the same
        // path through the remaining tiles and their barriers.
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        ok = __syncthreads_and(ok ? 1 : 0) != 0;
        ok = ok && !*bfail;

        // ---- η_i = Σ_j δ_ij u_j
        cx<float> u[M];
#pragma unroll
        for (int j = 0; j < M; j++) u[j] = ut[(size_t)j * N + t];
#pragma unroll
        for (int i = 0; i < M; i++) {
            float er = 0.f, ei = 0.f;
#pragma unroll
            for (int j = 0; j < M; j++) {
                er += dv[i * M + j] * u[j].re;
                ei += dv[i * M + j] * u[j].im;
            }
            eta[(size_t)i * N + t] = ok ? mk(er, ei) : mk(__int_as_float(0x7fc00000), 0.f);
        }
    }

    // ---- a B copy not waited for (no tile) or timed out may still be in
    // flight: wait for it (bounded) before the CTA's shared memory is released
    if (tid == 0 && (!b_waited || *bfail)) {
        uint32_t got = 0;
        for (long it = 0; it < (1L << 26) && !got; it++) {
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(got)
                : "r"(smem_u32(bbar))
                : "memory");
        }
    }
    // ---- MMAs whose completion wait timed out may still be writing tensor
    // memory: no later tile issued any (ok stays false), so the commit of
    // that tile is the last one; wait for its arrival before the
    // deallocation (a second, longer bound).  MMAs finish in microseconds,
    // so this only runs after a fault elsewhere; should even this wait give
    // up, the memory is released all the same, because a CTA that exits
    // holding tensor memory can block later allocations on its SM.
    if (tid == 0 && mma_pending >= 0) {
        uint32_t got = 0;
        for (long it = 0; it < (1L << 30) && !got; it++) {
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(got)
                : "r"(smem_u32(mbar)), "r"((uint32_t)mma_pending)
                : "memory");
        }
    }
    // ---- release tensor memory
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot),
                     "r"(128));
}

// ---------------------------------------------------------------------------
// Adjoint assembly of FP32-forward batches (M >= 6).  Per time point the
// FP64 assembly (sensitivity_disp_mmf.jl:94-140)
//   η_j = Σ_q S'_q g_qj - (1-fR) Σ_q w_q conj(g_qj) + 2i Σ_i C_ij u_i,
//   g_qj = Σ_i λ_i G[i,j,q],   w_q = u_k u_l  (q = (k, l), k <= l)
// regroups, G being real, into
//   η_j = Σ_i [λ_i D'_ij - (1-fR) conj(λ_i) W_ij] + 2i Σ_i C_ij u_i,
//   D'_ij = Σ_q G[i,j,q] S'_q,   W_ij = Σ_q G[i,j,q] w_q.
// D' and W depend on the forward field alone, which the FP32 forward knows
// to FP32 accuracy: they are three GEMMs of the forward contraction's shape
// (A = S', Re w, Im w over a 128-point tile; B = G) on the tensor cores in
// 3xTF32, while λ, C and the sums over i stay in FP64.  This takes the
// assembly from about 14 300 FP64 FMAs per time point (10 modes) to 800.
//
// G is symmetric in (i, j), so D' and W are too: B holds only the pairs
// p = (i <= j) (rows padded to 16, the symmetric image), each accumulator
// is NS <= 64 columns and the three fit a 256-column allocation.  With one
// A buffer (the three A tiles in turn, each after the previous MMAs have
// completed) a CTA takes 87 KB of shared memory at M = 10: two CTAs per SM,
// each one's loads overlapping the other's tensor-core and drain phases.
// Waits are bounded as in the forward contraction (a timeout sets the
// tile's outputs to NaN) and tensor memory is freed on every path.
template <int M>
struct TcSymShape {
    static constexpr int NP = M * (M + 1) / 2;
    static constexpr int KP = tc_kp(M);
    static constexpr int NS = (NP + 15) & ~15;          // MMA N: the pairs i <= j
    static constexpr int CS = (NS + 31) & ~31;          // columns between accumulators
    static constexpr int A_BYTES = kTcRows * KP * 4;    // one of A_hi / A_lo
    static constexpr int B_BYTES = NS * KP * 4;         // one of B_hi / B_lo
    static constexpr int U_BYTES = NS * mm_krmax(M) * 4;  // low-rank form: one of U_hi / U_lo
    static constexpr int SMEM = 2 * A_BYTES + 2 * B_BYTES + 2 * U_BYTES + 64 + 1024;
    // at least 80 KB so that no more than two CTAs (2 x 256 tensor-memory
    // columns) share an SM: no allocation waits on another CTA's
    static constexpr int SMEM_LAUNCH = SMEM > 80 * 1024 ? SMEM : 80 * 1024;
    static constexpr uint32_t TMEM_COLS = 256;
    static_assert(NS <= 256, "MMA N");
    static_assert(4 * CS <= (int)TMEM_COLS, "accumulator columns (four in the low-rank form)");
    static_assert(2 * SMEM <= 227 * 1024, "two CTAs per SM");
};

__host__ __device__ constexpr uint32_t tc_sym_bytes(int M) {
    return 2u * (uint32_t)(((M * (M + 1) / 2 + 15) & ~15) * tc_kp(M) * 4);
}

// bounded wait on an mbarrier phase (true: the phase completed)
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, long bound) {
    uint32_t done = 0;
    for (long it = 0; it < bound && !done; it++) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
    }
    return done != 0;
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, "
        "%9, %10, %11, %12, %13, %14, %15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}

// One A tile (this thread's row = time point) in the K-major layout, split
// TF32 hi/lo: column q = pair (k, l) holds f(q, k, l); zeros for q >= NP.
template <int M, int KP, class F>
__device__ __forceinline__ void tc_fill_pairs(unsigned char* Ahi, unsigned char* Alo, F&& f) {
    const int tid = threadIdx.x;
    float h[4], l[4];
    int q = 0;
#pragma unroll
    for (int k = 0; k < M; k++) {
#pragma unroll
        for (int k2 = k; k2 < M; k2++) {
            const float x = f(q, k, k2);
            h[q & 3] = tf32_rn(x);
            l[q & 3] = tf32_rn(x - h[q & 3]);
            if ((q & 3) == 3) {
                *reinterpret_cast<float4*>(Ahi + tc_off<KP>(tid, q - 3)) = make_float4(h[0], h[1], h[2], h[3]);
                *reinterpret_cast<float4*>(Alo + tc_off<KP>(tid, q - 3)) = make_float4(l[0], l[1], l[2], l[3]);
            }
            q++;
        }
    }
#pragma unroll
    for (int r = M * (M + 1) / 2; r < KP; r++) {
        h[r & 3] = 0.f;
        l[r & 3] = 0.f;
        if ((r & 3) == 3) {
            *reinterpret_cast<float4*>(Ahi + tc_off<KP>(tid, r - 3)) = make_float4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<float4*>(Alo + tc_off<KP>(tid, r - 3)) = make_float4(l[0], l[1], l[2], l[3]);
        }
    }
}

// the adjoint assembly's A tiles: op 0 = S'_q, op 1 = Re w_q, op 2 = Im w_q
template <int M, int KP>
__device__ __forceinline__ void tc_adj_fill(int op, unsigned char* Ahi, unsigned char* Alo,
                                            const float* __restrict__ sq, size_t N, int t,
                                            const cx<float> (&uf)[M]) {
    tc_fill_pairs<M, KP>(Ahi, Alo, [&](int q, int k, int l) -> float {
        if (op == 0) return sq[(size_t)q * N + t];
        const cx<float> w = cmul(uf[k], uf[l]);
        return op == 1 ? w.re : w.im;
    });
}

// The adjoint assembly of the 128-point tile `tile` of one slot.
template <int M>
__device__ void mm_contract_adj_tc(const MmDesc& d, int tile, unsigned char* smem) {
    using TS = TcSymShape<M>;
    constexpr int KP = TS::KP, NS = TS::NS, CS = TS::CS;
    static_assert(KP % 4 == 0, "float4 groups");
    const size_t N = (size_t)d.N;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int t = tile * kTcRows + tid;
    unsigned char* base =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem) + 1023) & ~uintptr_t(1023));
    unsigned char* Ahi = base;
    unsigned char* Alo = Ahi + TS::A_BYTES;
    unsigned char* Bhi = Alo + TS::A_BYTES;
    unsigned char* Blo = Bhi + TS::B_BYTES;
    unsigned char* Uhi = Blo + TS::B_BYTES;  // low-rank form: U (rows p, kr deep)
    uint64_t* bars = reinterpret_cast<uint64_t*>(Uhi + 2 * TS::U_BYTES);  // MMAs, B images
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
    uint32_t* bfail = tmem_slot + 1;
    const uint32_t barM = smem_u32(bars), barB = smem_u32(bars + 1);
    // the low-rank form takes D' = U S̃' (K = the rank, padded to 8)
    const int kr = d.rank > 0 ? (d.rank + 7) & ~7 : 0;
    const uint32_t u_bytes = (uint32_t)NS * kr * 4;
    unsigned char* Ulo = Uhi + u_bytes;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(TS::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    constexpr uint32_t kBBytes = 2 * TS::B_BYTES, kBChunk = 16384;
    static_assert(kBBytes % 16 == 0, "bulk copy size");
    if (tid == 0) {
        *bfail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barM));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barB));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(barB),
                     "r"(kBBytes + 2 * u_bytes)
                     : "memory");
        for (int img = 0; img < 2; img++) {  // G (symmetric), then U if used
            const char* src = reinterpret_cast<const char*>(img == 0 ? d.Gtcs : d.Utcs);
            const uint32_t bytes = img == 0 ? kBBytes : 2 * u_bytes;  // multiples of 16
            const uint32_t dst = smem_u32(img == 0 ? Bhi : Uhi);
            for (uint32_t off = 0; off < bytes; off += kBChunk) {
                const uint32_t n = bytes - off < kBChunk ? bytes - off : kBChunk;
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], "
                    "%2, [%3];" ::"r"(dst + off),
                    "l"(src + off), "r"(n), "r"(barB)
                    : "memory");
            }
        }
    }

    // the mixed adjoint's FP32 forward field and S' (the FP32 kernels' output)
    const float* sq = static_cast<const float*>(d.sq);
    const double* cq = static_cast<const double*>(d.cq);
    const cx<float>* ut = static_cast<const cx<float>*>(d.ut);
    const cx<double>* lt = static_cast<const cx<double>*>(d.lt);
    cx<double>* eta = static_cast<cx<double>*>(d.eta);
    cx<float> uf[M];
#pragma unroll
    for (int i = 0; i < M; i++) uf[i] = ut[(size_t)i * N + t];

    // ---- the A tiles in turn: S' (or S̃') -> columns [0, NS), Re w -> [CS,
    // CS + NS), Im w -> [2 CS, 2 CS + NS) and, in the low-rank form, the
    // correlations Cz -> [3 CS, 3 CS + NS) (C = U Cz); each refill waits for
    // the MMAs that read the previous tile (barrier phases 0, 1, 0, 1)
    const uint32_t bh = smem_u32(Bhi), bl = smem_u32(Blo);
    const int nops = kr > 0 ? 4 : 3;
    uint32_t tmem = 0;
    bool ok = true;
    int pending = -1;  // parity of a commit whose arrival a timed-out wait did not see
#pragma unroll 1
    for (int op = 0; op < nops; op++) {
        if (op > 0) {  // wait for the previous tile's MMAs (block-uniform outcome)
            const bool done = tc_wait(barM, (uint32_t)((op - 1) & 1), 1L << 26);
            if (!done && pending < 0) pending = (op - 1) & 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            ok = __syncthreads_and(ok && done ? 1 : 0) != 0;
            if (!ok) break;
        }
        const bool lowrank = (op == 0 || op == 3) && kr > 0;
        if (lowrank) {
            // A = S̃'_k or Cz_k (k < rank), kr deep
#pragma unroll 2
            for (int k = 0; k < kr; k += 4) {
                float4 hi, lo;
                float* h = &hi.x;
                float* l = &lo.x;
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const float x = k + c >= d.rank ? 0.f
                                    : op == 0       ? sq[(size_t)(k + c) * N + t]
                                                    : (float)cq[(size_t)(k + c) * N + t];
                    h[c] = tf32_rn(x);
                    l[c] = tf32_rn(x - h[c]);
                }
                *reinterpret_cast<float4*>(Ahi + tc_off_rt(tid, k, kr)) = hi;
                *reinterpret_cast<float4*>(Alo + tc_off_rt(tid, k, kr)) = lo;
            }
        } else {
            tc_adj_fill<M, KP>(op, Ahi, Alo, sq, N, t, uf);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tmem = *tmem_slot;
        if (tid == 0) {
            if (op == 0 && !tc_wait(barB, 0, 1L << 26)) *bfail = 1;
            if (!*bfail) {
                if (lowrank)
                    tc_issue3(tmem + (uint32_t)(op * CS), smem_u32(Ahi), smem_u32(Alo), smem_u32(Uhi),
                              smem_u32(Ulo), kr, NS);
                else
                    tc_issue3(tmem + (uint32_t)(op * CS), smem_u32(Ahi), smem_u32(Alo), bh, bl, KP, NS);
            }
            tc_commit(barM);  // arrives once the MMAs above (if any) have completed
        }
    }

    // ---- η_j = 2i Σ_i C_ij u_i + Σ_i [λ_i D'_ij - (1-fR) conj(λ_i) W_ij]; the
    // FP64 loads and the C term run while the tensor cores finish
    cx<double> la[M];
#pragma unroll
    for (int i = 0; i < M; i++) la[i] = lt[(size_t)i * N + t];
    double er[M], ei[M];
    {
        cx<double> u[M];
#pragma unroll
        for (int i = 0; i < M; i++) {
            u[i] = mk((double)uf[i].re, (double)uf[i].im);
            er[i] = 0.0;
            ei[i] = 0.0;
        }
        if (kr == 0) {  // (the low-rank form reads C from tensor memory below)
            int p = 0;
#pragma unroll
            for (int a = 0; a < M; a++) {
#pragma unroll
                for (int b = a; b < M; b++) {
                    const double c2 = 2.0 * cq[(size_t)p * N + t];
                    er[b] -= c2 * u[a].im;
                    ei[b] += c2 * u[a].re;
                    if (a != b) {
                        er[a] -= c2 * u[b].im;
                        ei[a] += c2 * u[b].re;
                    }
                    p++;
                }
            }
        }
    }
    if (ok) {  // the last tile's MMAs
        const uint32_t par = (uint32_t)((nops - 1) & 1);
        const bool done = tc_wait(barM, par, 1L << 26);
        if (!done && pending < 0) pending = (int)par;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        ok = __syncthreads_and(done ? 1 : 0) != 0;
    }
    ok = ok && !*bfail;

    if (ok) {
        const double ofr = d.one_m_fR;
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        float Dv[16], Wr[16], Wi[16], Cv[16];
        int p = 0;
#pragma unroll
        for (int a = 0; a < M; a++) {
#pragma unroll
            for (int b = a; b < M; b++) {
                if ((p & 15) == 0) {  // the next 16 pairs of each accumulator
                    tc_ld16(trow + (uint32_t)p, Dv);
                    tc_ld16(trow + (uint32_t)(CS + p), Wr);
                    tc_ld16(trow + (uint32_t)(2 * CS + p), Wi);
                    if (kr > 0) tc_ld16(trow + (uint32_t)(3 * CS + p), Cv);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                }
                if (kr > 0) {  // 2i C_ab u_a into η_b (and the mirror)
                    const double c2 = 2.0 * (double)Cv[p & 15];
                    er[b] -= c2 * (double)uf[a].im;
                    ei[b] += c2 * (double)uf[a].re;
                    if (a != b) {
                        er[a] -= c2 * (double)uf[b].im;
                        ei[a] += c2 * (double)uf[b].re;
                    }
                }
                const double dv = Dv[p & 15], wr = Wr[p & 15], wi = Wi[p & 15];
                // η_b += λ_a D'_ab - (1-fR) conj(λ_a) W_ab, and (a != b) the mirror
                er[b] += la[a].re * dv - ofr * (la[a].re * wr + la[a].im * wi);
                ei[b] += la[a].im * dv - ofr * (la[a].re * wi - la[a].im * wr);
                if (a != b) {
                    er[a] += la[b].re * dv - ofr * (la[b].re * wr + la[b].im * wi);
                    ei[a] += la[b].im * dv - ofr * (la[b].re * wi - la[b].im * wr);
                }
                p++;
            }
        }
    }
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
    for (int j = 0; j < M; j++) eta[(size_t)j * N + t] = ok ? mk(er[j], ei[j]) : mk(nan, 0.0);

    // ---- cleanup: a B copy that timed out, or MMAs whose completion a
    // timed-out wait did not see (no MMA was issued after it), may still be
    // in flight: wait for them (bounded) before shared and tensor memory are
    // released
    if (tid == 0) {
        if (*bfail) tc_wait(barB, 0, 1L << 26);
        if (pending >= 0) tc_wait(barM, (uint32_t)pending, 1L << 30);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot),
                     "r"(TS::TMEM_COLS));
}

// ---------------------------------------------------------------------------
// Adjoint first pass of FP32-forward batches (M >= 6) on the tensor cores:
//   Im X_p = Σ_q G[i,j,q] Y_q  for the pairs p = (i <= j),
//   Y_q = (Im(λ_k u_l*) + Im(λ_l u_k*))/2 (k < l), Im(λ_k u_k*) (k = l),
// one GEMM with A = Y (formed in FP64, split 3xTF32) and the symmetric B
// image (rows p): column p of each thread's accumulator row is Im X_p,
// stored to C's input table in FP64.  Waits are bounded (a timeout writes
// NaN) and tensor memory is freed on every path.
template <int M>
__device__ void mm_imx_tc(const MmDesc& d, int tile, unsigned char* smem) {
    using TS = TcSymShape<M>;
    constexpr int KP = TS::KP, NS = TS::NS, NP = TS::NP;
    constexpr uint32_t kCols = NS <= 32 ? 32 : NS <= 64 ? 64 : 128;  // allocation: a power of 2 >= 32
    const size_t N = (size_t)d.N;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int t = tile * kTcRows + tid;
    unsigned char* base =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem) + 1023) & ~uintptr_t(1023));
    unsigned char* Ahi = base;
    unsigned char* Alo = Ahi + TS::A_BYTES;
    unsigned char* Bhi = Alo + TS::A_BYTES;
    // the low-rank form reduces Y to the rank instead: Yz_k = Σ_q V[q][k] Y_q
    // (B = the V image, rows k), whose correlations the pair kernel takes
    const bool lr = d.rank > 0;
    const int nb = lr ? (d.rank + 15) & ~15 : NS, nout = lr ? d.rank : NP;
    const uint32_t b_bytes = (uint32_t)nb * KP * 4;
    unsigned char* Blo = Bhi + b_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(Bhi + 2 * TS::B_BYTES);  // MMAs, B image
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
    uint32_t* bfail = tmem_slot + 1;
    const uint32_t barM = smem_u32(bars), barB = smem_u32(bars + 1);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    const uint32_t kBBytes = 2 * b_bytes, kBChunk = 16384;  // a multiple of 16
    if (tid == 0) {
        *bfail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barM));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barB));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(barB),
                     "r"(kBBytes)
                     : "memory");
        const char* src = reinterpret_cast<const char*>(lr ? d.Vz : d.Gtcs);
        for (uint32_t off = 0; off < kBBytes; off += kBChunk) {
            const uint32_t n = kBBytes - off < kBChunk ? kBBytes - off : kBChunk;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
                "[%3];" ::"r"(smem_u32(Bhi) + off),
                "l"(src + off), "r"(n), "r"(barB)
                : "memory");
        }
    }
    const cx<double>* lt = static_cast<const cx<double>*>(d.lt);
    const cx<float>* ut = static_cast<const cx<float>*>(d.ut);  // the mixed adjoint's FP32 field
    double* cq = static_cast<double*>(d.cq);
    cx<double> la[M], u[M];
#pragma unroll
    for (int i = 0; i < M; i++) {
        la[i] = lt[(size_t)i * N + t];
        const cx<float> x = ut[(size_t)i * N + t];
        u[i] = mk((double)x.re, (double)x.im);
    }
    tc_fill_pairs<M, KP>(Ahi, Alo, [&](int, int k, int l) -> float {
        const double a = la[k].im * u[l].re - la[k].re * u[l].im;  // Im(λ_k u_l*)
        if (k == l) return (float)a;
        const double b = la[l].im * u[k].re - la[l].re * u[k].im;
        return (float)(0.5 * (a + b));
    });
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    if (tid == 0) {
        if (!tc_wait(barB, 0, 1L << 26)) *bfail = 1;
        if (!*bfail) tc_issue3(tmem, smem_u32(Ahi), smem_u32(Alo), smem_u32(Bhi), smem_u32(Blo), KP, nb);
        tc_commit(barM);
    }
    const bool done = tc_wait(barM, 0, 1L << 26);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool ok = __syncthreads_and(done ? 1 : 0) != 0 && !*bfail;
    if (ok) {
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c = 0; c < nb; c += 16) {
            float v[16];
            tc_ld16(trow + (uint32_t)c, v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int e = 0; e < 16; e++)
                if (c + e < nout) cq[(size_t)(c + e) * N + t] = (double)v[e];
        }
    } else {
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll 1
        for (int p = 0; p < nout; p++) cq[(size_t)p * N + t] = nan;
    }
    if (tid == 0) {
        if (*bfail) tc_wait(barB, 0, 1L << 26);
        if (!done) tc_wait(barM, 0, 1L << 30);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot),
                     "r"(kCols));
}

// ---------------------------------------------------------------------------
// The low-rank form's reduction (rank > 0): Z_k = Σ_q V[q][k] P_q over the
// pair products P_q = Re(u_k' u_l'*) of the FP32 forward field, for the
// forward and the mixed adjoint alike, one GEMM per 128-point tile with A = P
// (split 3xTF32) and B = the V image (rows k, the rank padded to 16).  The
// pair transforms then convolve the Z_k (upper half of the pair table, FP32
// rows) instead of the NP products.  In the adjoint the same kernel reduces
// Y (the Im X inputs) to the rank with a second GEMM on the same image.
// Waits are bounded (a timeout writes NaN) and tensor memory is freed on
// every path.
template <int M>
__device__ void mm_z_tc(const MmDesc& d, int tile, unsigned char* smem, bool adj) {
    using TS = TcShape<M>;
    constexpr int KP = TS::KP, NP = TS::NP;
    constexpr uint32_t kCols = 64;  // Z in [0, 32), the adjoint's Yz in [32, 64)
    static_assert(((mm_krmax(M) + 15) & ~15) <= 32, "Z accumulator columns");
    const size_t N = (size_t)d.N;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int t = tile * kTcRows + tid;
    const int r = d.rank, nz = (r + 15) & ~15;
    unsigned char* base =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem) + 1023) & ~uintptr_t(1023));
    unsigned char* Ahi = base;
    unsigned char* Alo = Ahi + TS::A_BYTES;
    unsigned char* Bhi = Alo + TS::A_BYTES;
    const uint32_t b_bytes = (uint32_t)nz * KP * 4;
    unsigned char* Blo = Bhi + b_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(Bhi + 2 * TS::B_BYTES);  // MMAs, B image
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
    uint32_t* bfail = tmem_slot + 1;
    const uint32_t barM = smem_u32(bars), barB = smem_u32(bars + 1);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    const uint32_t kBBytes = 2 * b_bytes, kBChunk = 16384;  // a multiple of 16
    if (tid == 0) {
        *bfail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barM));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barB));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(barB),
                     "r"(kBBytes)
                     : "memory");
        const char* src = reinterpret_cast<const char*>(d.Vz);
        for (uint32_t off = 0; off < kBBytes; off += kBChunk) {
            const uint32_t n = kBBytes - off < kBChunk ? kBBytes - off : kBChunk;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
                "[%3];" ::"r"(smem_u32(Bhi) + off),
                "l"(src + off), "r"(n), "r"(barB)
                : "memory");
        }
    }
    const cx<float>* ut = static_cast<const cx<float>*>(d.ut);
    float* zq = static_cast<float*>(d.sq) + (size_t)NP * N;  // upper half of the pair table
    cx<float> u[M];
#pragma unroll
    for (int i = 0; i < M; i++) u[i] = ut[(size_t)i * N + t];
    tc_fill_pairs<M, KP>(Ahi, Alo, [&](int, int k, int l) -> float {
        return u[k].re * u[l].re + u[k].im * u[l].im;  // Re(u_k u_l*)
    });
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    if (tid == 0) {
        if (!tc_wait(barB, 0, 1L << 26)) *bfail = 1;
        if (!*bfail) tc_issue3(tmem, smem_u32(Ahi), smem_u32(Alo), smem_u32(Bhi), smem_u32(Blo), KP, nz);
        tc_commit(barM);
    }
    bool done = tc_wait(barM, 0, 1L << 26);
    int pending = done ? -1 : 0;  // parity of a commit whose arrival a timed-out wait did not see
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    bool ok = __syncthreads_and(done ? 1 : 0) != 0;
    // the adjoint also reduces Y_q = (Im(λ_k u_l*) + Im(λ_l u_k*))/2 (k < l),
    // Im(λ_k u_k*) (k = l) to Yz_k = Σ_q V[q][k] Y_q (columns [32, 32 + nz)),
    // whose correlations the FP64 pair kernel takes (C = U Cz)
    if (adj && ok) {
        const cx<double>* lt = static_cast<const cx<double>*>(d.lt);
        cx<double> la[M];
#pragma unroll
        for (int i = 0; i < M; i++) la[i] = lt[(size_t)i * N + t];
        tc_fill_pairs<M, KP>(Ahi, Alo, [&](int, int k, int l) -> float {
            const double a = la[k].im * (double)u[l].re - la[k].re * (double)u[l].im;  // Im(λ_k u_l*)
            if (k == l) return (float)a;
            const double b = la[l].im * (double)u[k].re - la[l].re * (double)u[k].im;
            return (float)(0.5 * (a + b));
        });
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            if (!*bfail)
                tc_issue3(tmem + 32, smem_u32(Ahi), smem_u32(Alo), smem_u32(Bhi), smem_u32(Blo), KP, nz);
            tc_commit(barM);
        }
        done = tc_wait(barM, 1, 1L << 26);
        if (!done) pending = 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        ok = __syncthreads_and(done ? 1 : 0) != 0;
    }
    ok = ok && !*bfail;
    double* cq = static_cast<double*>(d.cq);
    if (ok) {
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c = 0; c < nz; c += 16) {
            float v[16];
            tc_ld16(trow + (uint32_t)c, v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int e = 0; e < 16; e++)
                if (c + e < r) zq[(size_t)(c + e) * N + t] = v[e];
            if (adj) {
                tc_ld16(trow + (uint32_t)(32 + c), v);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int e = 0; e < 16; e++)
                    if (c + e < r) cq[(size_t)(c + e) * N + t] = (double)v[e];
            }
        }
    } else {
#pragma unroll 1
        for (int k = 0; k < r; k++) {
            zq[(size_t)k * N + t] = __int_as_float(0x7fc00000);
            if (adj) cq[(size_t)k * N + t] = __longlong_as_double(0x7ff8000000000000LL);
        }
    }
    if (tid == 0) {
        if (*bfail) tc_wait(barB, 0, 1L << 26);
        if (pending >= 0) tc_wait(barM, (uint32_t)pending, 1L << 30);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot),
                     "r"(kCols));
}

}  // namespace fl
