// fl_tc.cuh -- forward Kerr/Raman contraction of the multimode stepper on the
// 5th-generation tensor cores (tcgen05, sm_100a), for M >= 6 modes.
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
// (128 columns) and freed before the CTA exits on every path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

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

// The forward contraction of the 128-point tiles t0 = tile*128, tile =
// first, first + step, ... < N/128 of one slot.  The B operand (the G table,
// split hi/lo) and the tensor memory are set up once per CTA; each tile
// refills A, issues its MMAs and waits on the barrier's next phase.
template <int M>
__device__ void mm_contract_fwd_tc(const MmDesc& d, int first, int step, unsigned char* smem) {
    using TS = TcShape<M>;
    constexpr int NP = TS::NP, KP = TS::KP, GP = TS::GP, NN = TS::NN;
    const int N = d.N, ntiles = N / kTcRows;
    const int tid = threadIdx.x, warp = tid >> 5;
    (void)GP;
    // 1024-byte aligned operand area
    unsigned char* base =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem) + 1023) & ~uintptr_t(1023));
    unsigned char* Ahi = base;
    unsigned char* Alo = Ahi + TS::A_BYTES;
    unsigned char* Bhi = Alo + TS::A_BYTES;
    unsigned char* Blo = Bhi + TS::B_BYTES;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(Blo + TS::B_BYTES);  // MMA completion
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
    constexpr uint32_t kBBytes = 2 * TS::B_BYTES, kBChunk = 16384;
    static_assert(kBBytes % 16 == 0, "bulk copy size");
    if (tid == 0) {
        *bfail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                         smem_u32(bbar)),
                     "r"(kBBytes)
                     : "memory");
        const char* src = reinterpret_cast<const char*>(d.Gtc);
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
        // ---- A = this tile's S, split hi/lo: four pairs per 16-byte store
#pragma unroll 2
        for (int k = 0; k < KP; k += 4) {
            float4 hi, lo;
            float* h = &hi.x;
            float* l = &lo.x;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const float s = k + c < NP ? sq[(size_t)(k + c) * N + t] : 0.f;
                h[c] = tf32_rn(s);
                l[c] = tf32_rn(s - h[c]);
            }
            *reinterpret_cast<float4*>(Ahi + tc_off<KP>(tid, k)) = hi;
            *reinterpret_cast<float4*>(Alo + tc_off<KP>(tid, k)) = lo;
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
        if (tid == 0 && !*bfail) {
            constexpr uint32_t idesc = tc_idesc(NN);
            const uint32_t a_hi = smem_u32(Ahi), a_lo = smem_u32(Alo);
            const uint32_t b_hi = smem_u32(Bhi), b_lo = smem_u32(Blo);
#pragma unroll
            for (int ks = 0; ks < KP / 8; ks++) {
                const uint32_t koff = (uint32_t)ks * 256;
                const uint64_t dah = tc_desc(a_hi + koff, 128, TS::SBO);
                const uint64_t dal = tc_desc(a_lo + koff, 128, TS::SBO);
                const uint64_t dbh = tc_desc(b_hi + koff, 128, TS::SBO);
                const uint64_t dbl = tc_desc(b_lo + koff, 128, TS::SBO);
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

}  // namespace fl
