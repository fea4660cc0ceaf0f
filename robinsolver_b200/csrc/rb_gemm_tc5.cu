// rb_gemm_tc5.cu -- descriptor-batched complex GEMM on the 5th-generation tensor cores
// (tcgen05.mma kind::tf32, FP32 accumulators in tensor memory), for the mixed-precision factor
// and solve of the lower merge levels.
//
// Split TF32 ("TF32x3"): every FP64 operand element x is held as two TF32 numbers,
// hi = tf32(x) and lo = tf32(x - hi), so x = hi + lo to about 22 significant bits, and a real
// product a*b is taken as ah*bh + ah*bl + al*bh (the lo*lo term is below that precision).  A
// complex product is four real ones (re*re - im*im, re*im + im*re); the minus sign is the MMA's
// own A-negate bit, so no negated copy of an operand is stored.  Twelve tcgen05.mma per k-step
// of 8 accumulate into two FP32 accumulators in tensor memory, Cr and Ci (128 lanes x BN
// columns each).  The result carries ~1e-6 relative error: the solve recovers FP64 accuracy by
// iterative refinement against the FP64 residual (rb_refine.cu).
//
// CTA = one 128 x BN output tile of one problem (blockIdx.y), 9 warps:
//   warps 0-7  producers: cp.async (16 bytes, zero-filled outside the problem) of the FP64 operands
//              through the problem's ZViews (face gathers, row maps, skipped bands, exactly as the
//              FP64 kernels) into a ring of STAGES shared-memory stages, STAGES - 1 k-blocks ahead of
//              the one being converted.  A landed stage is split to TF32 hi/lo IN PLACE (the four
//              TF32 parts of an element take the 16 bytes of its FP64 pair) into the UMMA K-major
//              no-swizzle layout, then handed to the MMA warp.  Then the epilogue: tcgen05.ld of
//              the accumulators (warp w reads lanes 32 (w % 4) .. +31, half w / 4 of the columns),
//              alpha/beta, scatter through the output maps.
//   warp 8     allocates 2*BN tensor-memory columns; one lane issues the MMAs of each stage once
//              its producers have arrived, and releases the stage with tcgen05.commit.
// Every mbarrier wait is bounded (RB_TC5_WAIT_NS on the global timer).  A wait that runs out sets
// RB_TC5_TIMEOUT in the status word, the CTA stops issuing work, waits (bounded) for the MMAs it
// issued, frees its tensor memory and returns.
#include <algorithm>
#include <cstdint>

#include "rb_kernels.h"

namespace rb {

namespace {

constexpr int TC5_BM = 128;          // output rows per tile = UMMA M (one lane per row)
constexpr int TC5_KB = 16;           // complex k per stage: 4 chunks of 4 TF32 = two UMMA k-steps
constexpr int TC5_PRODUCERS = 256;   // warps 0-7
constexpr int TC5_THREADS = TC5_PRODUCERS + 32;
constexpr unsigned long long RB_TC5_WAIT_NS = 1000000000ull;   // 1 s per wait

template <int BN>
struct Tc5Cfg {
    // one stage: A (128 rows x KB complex) then B (BN columns x KB complex), 16 bytes per element;
    // raw FP64 pairs first, the four TF32 parts (re/im x hi/lo) in the same bytes after the split
    static constexpr int A_BYTES = TC5_BM * TC5_KB * 16;
    static constexpr int B_BYTES = BN * TC5_KB * 16;
    static constexpr int A_PART = TC5_BM * TC5_KB * 4;     // one TF32 part of A
    static constexpr int B_PART = BN * TC5_KB * 4;
    static constexpr int STAGE = A_BYTES + B_BYTES;
    static constexpr int STAGES = (196608 / STAGE) < 4 ? (196608 / STAGE) : 4;   // 3 (BN 128) or 4
    static constexpr int AHEAD = STAGES - 1;               // k-blocks in flight beyond the converted one
    // + 1024 for the alignment of the stages
    static constexpr int SMEM = STAGES * STAGE + 1024;
    static constexpr int TMEM_COLS = 2 * BN;               // Cr, Ci
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.release.cta.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar)
        : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// waits for the phase with the given parity to complete; false after RB_TC5_WAIT_NS or when
// another warp has already given up (*abort)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned it = 0;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 63) == 63) {
            if (*abort) return false;
            if (global_ns() - t0 > RB_TC5_WAIT_NS) return false;
        }
    }
}

__device__ __forceinline__ uint32_t tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// x -> (hi, lo): hi = tf32(x), lo = tf32(x - hi) with the difference taken in FP64
__device__ __forceinline__ void split_tf32(double x, uint32_t& hi, uint32_t& lo) {
    hi = tf32_rna(static_cast<float>(x));
    lo = tf32_rna(static_cast<float>(x - static_cast<double>(__uint_as_float(hi))));
}

// UMMA shared-memory descriptor, K-major, no swizzle: core matrices of 8 rows x 16 bytes, rows
// 16 bytes apart; sbo = bytes between 8-row groups, lbo = bytes between the two 16-byte K chunks
// of one k-step.  Version 1 (sm_100), base offset 0, layout type 0 (SWIZZLE_NONE).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor of kind::tf32: D FP32, A and B TF32, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t tc5_idesc(int n, bool neg_a) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(TC5_BM >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    // src-size 0 fills the 16 bytes with zeros (a row, column or k outside the problem)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
// the 256 producer threads only (the MMA warp runs its own loop)
__device__ __forceinline__ void producers_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }
// a producer barrier that also ORs a flag over the 256 producers: every one gets the same answer,
// so they all leave the loop at the same iteration
__device__ __forceinline__ bool producers_any(bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, 256, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void split4(const z (&v)[4], uint4& rh, uint4& rl, uint4& ih, uint4& il) {
    split_tf32(v[0].x, rh.x, rl.x); split_tf32(v[0].y, ih.x, il.x);
    split_tf32(v[1].x, rh.y, rl.y); split_tf32(v[1].y, ih.y, il.y);
    split_tf32(v[2].x, rh.z, rl.z); split_tf32(v[2].y, ih.z, il.z);
    split_tf32(v[3].x, rh.w, rl.w); split_tf32(v[3].y, ih.w, il.w);
}

}  // namespace

// Split-K (part != nullptr): blockIdx.z takes k in [z * kchunk, (z + 1) * kchunk) and writes its raw
// sums to part + (problem * ksplit + z) * pstride + i + j * ldp; the reduction kernel finishes.
template <int BN>
__global__ void __launch_bounds__(TC5_THREADS, 1) zgemm_tc5_kernel(const GemmDesc* __restrict__ descs, int* status,
                                                                  int kchunk, z* part, long long pstride, int ldp,
                                                                  int ksplit) {
    using Cfg = Tc5Cfg<BN>;
    constexpr int STAGES = Cfg::STAGES;
    extern __shared__ __align__(1024) unsigned char tc5_smem[];
    __shared__ GemmDesc sd;
    __shared__ int a_rows[TC5_BM];          // row offsets of the tile's rows in A (-1: outside m)
    __shared__ long long b_cols[BN];        // column offsets of the tile's columns in B (-1: outside n)
    __shared__ __align__(8) unsigned long long bars[2 * STAGES + 1];
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(descs + blockIdx.y);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sd);
        for (int w = tid; w < (int)(sizeof(GemmDesc) / 8); w += TC5_THREADS) dst[w] = src[w];
    }
    __syncthreads();
    const int m = sd.m, n = sd.n;
    const int kbeg = part ? (int)blockIdx.z * kchunk : 0;
    const int K = part ? min(sd.k, kbeg + kchunk) : sd.k;             // this CTA's k runs over [kbeg, K)
    const int tiles_m = (m + TC5_BM - 1) / TC5_BM;
    const int tiles_n = (n + BN - 1) / BN;
    if ((int)blockIdx.x >= tiles_m * tiles_n || K <= kbeg) {
        // nothing to sum: a split range past this problem's k still owes its share of zeros
        if (part && (int)blockIdx.x < tiles_m * tiles_n) {
            const int m0 = (blockIdx.x % tiles_m) * TC5_BM, n0 = (blockIdx.x / tiles_m) * BN;
            z* pp = part + ((long long)blockIdx.y * ksplit + blockIdx.z) * pstride;
            for (int e = threadIdx.x; e < TC5_BM * BN; e += TC5_THREADS) {
                const int i = m0 + e % TC5_BM, j = n0 + e / TC5_BM;
                if (i < m && j < n) pp[i + (long long)j * ldp] = zmk(0.0, 0.0);
            }
        }
        return;      // uniform over the CTA
    }
    const int m0 = (blockIdx.x % tiles_m) * TC5_BM;
    const int n0 = (blockIdx.x / tiles_m) * BN;

    unsigned char* stage_base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(tc5_smem) + 1023) & ~uintptr_t(1023));
    const uint32_t full0 = smem_u32(&bars[0]);
    const uint32_t empty0 = smem_u32(&bars[STAGES]);
    const uint32_t done_bar = smem_u32(&bars[2 * STAGES]);

    for (int i = tid; i < TC5_BM; i += TC5_THREADS) {
        const int gi = m0 + i;
        a_rows[i] = gi < m ? vrow(sd.A, gi) : -1;
    }
    for (int j = tid; j < BN; j += TC5_THREADS) {
        const int gj = n0 + j;
        b_cols[j] = gj < n ? (long long)vcol(sd.B, gj) * sd.B.ld : -1;
    }
    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full0 + 8 * s, TC5_PRODUCERS);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 8) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"((uint32_t)Cfg::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const int nkb = (K - kbeg + TC5_KB - 1) / TC5_KB;

    if (warp == 8) {
        // ---------------- MMA issuer: one lane, the warp kept converged ----------------------
        const uint32_t id_pos = tc5_idesc(BN, false), id_neg = tc5_idesc(BN, true);
        const uint32_t c_re = tmem, c_im = tmem + BN;
        bool ok = true;
        for (int kb = 0; kb < nkb && ok; ++kb) {
            const int s = kb % STAGES;
            const uint32_t par = (uint32_t)((kb / STAGES) & 1);
            ok = __all_sync(0xffffffffu, mbar_wait(full0 + 8 * s, par, &abort_flag));
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (lane == 0) {
                const uint32_t st = smem_u32(stage_base + (size_t)s * Cfg::STAGE);
                const uint32_t a_rh = st, a_rl = st + Cfg::A_PART, a_ih = st + 2 * Cfg::A_PART,
                               a_il = st + 3 * Cfg::A_PART;
                const uint32_t bb = st + Cfg::A_BYTES;
                const uint32_t b_rh = bb, b_rl = bb + Cfg::B_PART, b_ih = bb + 2 * Cfg::B_PART,
                               b_il = bb + 3 * Cfg::B_PART;
                // K chunk c of A sits at + c * 128 * 16 bytes, of B at + c * BN * 16
                constexpr uint32_t LBO_A = TC5_BM * 16, LBO_B = BN * 16, SBO = 128;
#pragma unroll
                for (int q = 0; q < TC5_KB / 8; ++q) {
                    const uint32_t oa = q * 2 * LBO_A, ob = q * 2 * LBO_B;
                    const uint64_t Arh = umma_desc(a_rh + oa, LBO_A, SBO), Arl = umma_desc(a_rl + oa, LBO_A, SBO);
                    const uint64_t Aih = umma_desc(a_ih + oa, LBO_A, SBO), Ail = umma_desc(a_il + oa, LBO_A, SBO);
                    const uint64_t Brh = umma_desc(b_rh + ob, LBO_B, SBO), Brl = umma_desc(b_rl + ob, LBO_B, SBO);
                    const uint64_t Bih = umma_desc(b_ih + ob, LBO_B, SBO), Bil = umma_desc(b_il + ob, LBO_B, SBO);
                    const uint32_t acc = (kb > 0 || q > 0) ? 1u : 0u;
                    // Cr = Ar Br - Ai Bi, small terms first
                    umma_tf32(c_re, Arl, Brh, id_pos, acc);
                    umma_tf32(c_re, Arh, Brl, id_pos, 1u);
                    umma_tf32(c_re, Ail, Bih, id_neg, 1u);
                    umma_tf32(c_re, Aih, Bil, id_neg, 1u);
                    umma_tf32(c_re, Arh, Brh, id_pos, 1u);
                    umma_tf32(c_re, Aih, Bih, id_neg, 1u);
                    // Ci = Ar Bi + Ai Br
                    umma_tf32(c_im, Arl, Bih, id_pos, acc);
                    umma_tf32(c_im, Arh, Bil, id_pos, 1u);
                    umma_tf32(c_im, Ail, Brh, id_pos, 1u);
                    umma_tf32(c_im, Aih, Brl, id_pos, 1u);
                    umma_tf32(c_im, Arh, Bih, id_pos, 1u);
                    umma_tf32(c_im, Aih, Brh, id_pos, 1u);
                }
                umma_commit(empty0 + 8 * s);          // the stage is free once these MMAs are done
            }
            __syncwarp();
        }
        if (!ok) {
            abort_flag = 1;
            if (lane == 0) atomicOr(status, RB_TC5_TIMEOUT);
        }
        // the accumulators are complete (or, after a timeout, every issued MMA has finished) when
        // this arrives: commit tracks all prior MMAs of this thread
        if (lane == 0) umma_commit(done_bar);
        __syncwarp();
    } else {
        // ---------------- producers --------------------------------------------------------------
        const z* __restrict__ Ap = sd.A.p;
        const z* __restrict__ Bp = sd.B.p;
        const long long lda = sd.A.ld;
        // cp.async of k-block kb into stage s: A element (i, k) to A + (k * 128 + i) * 16 (consecutive
        // threads take consecutive rows: A is column-major), B element (k, j) to B + (j * KB + k) * 16
        // (consecutive threads take consecutive k of a column)
        auto issue = [&](int kb, int s) {
            const int k0 = kbeg + kb * TC5_KB;
            const uint32_t st = smem_u32(stage_base + (size_t)s * Cfg::STAGE);
#pragma unroll
            for (int q = 0; q < TC5_BM * TC5_KB / TC5_PRODUCERS; ++q) {
                const int e = tid + q * TC5_PRODUCERS;
                const int i = e % TC5_BM, kk = e / TC5_BM, k = k0 + kk;
                const int ro = a_rows[i];
                const bool v = ro >= 0 && k < K;
                const z* src = v ? Ap + ro + (long long)vcol(sd.A, k) * lda : Ap;
                cp_async16(st + (uint32_t)(kk * TC5_BM + i) * 16, src, v);
            }
#pragma unroll
            for (int q = 0; q < (BN * TC5_KB + TC5_PRODUCERS - 1) / TC5_PRODUCERS; ++q) {
                const int e = tid + q * TC5_PRODUCERS;
                if (e >= BN * TC5_KB) break;
                const int kk = e % TC5_KB, j = e / TC5_KB, k = k0 + kk;
                const long long co = b_cols[j];
                const bool v = co >= 0 && k < K;
                const z* src = v ? Bp + vrow(sd.B, k) + co : Bp;
                cp_async16(st + Cfg::A_BYTES + (uint32_t)(j * TC5_KB + kk) * 16, src, v);
            }
        };
        // the landed FP64 pairs of stage s -> TF32 parts in place: A unit (row i, K chunk c) and B
        // unit (column j, chunk c) read their 4 pairs, all producers pass a barrier, then write
        // part p of A at A + p * A_PART + c * 128 * 16 + i * 16 and of B at B + p * B_PART +
        // c * BN * 16 + j * 16 (16 bytes: the chunk's 4 TF32 values)
        auto convert = [&](int s) {
            unsigned char* st = stage_base + (size_t)s * Cfg::STAGE;
            unsigned char* sb = st + Cfg::A_BYTES;
            constexpr int AU = TC5_BM * (TC5_KB / 4) / TC5_PRODUCERS;             // 2
            constexpr int BT = BN * (TC5_KB / 4);
            constexpr int BU = (BT + TC5_PRODUCERS - 1) / TC5_PRODUCERS;           // 1 or 2
            z av[AU][4], bv[BU][4];
#pragma unroll
            for (int u = 0; u < AU; ++u) {
                const int unit = tid + u * TC5_PRODUCERS, i = unit % TC5_BM, c = unit / TC5_BM;
#pragma unroll
                for (int e = 0; e < 4; ++e) av[u][e] = *reinterpret_cast<const z*>(st + ((4 * c + e) * TC5_BM + i) * 16);
            }
#pragma unroll
            for (int u = 0; u < BU; ++u) {
                const int unit = tid + u * TC5_PRODUCERS, j = unit / 4, c = unit % 4;
                if (unit < BT) {
#pragma unroll
                    for (int e = 0; e < 4; ++e) bv[u][e] = *reinterpret_cast<const z*>(sb + (j * TC5_KB + 4 * c + e) * 16);
                }
            }
            producers_sync();                    // every pair of the stage is read before any write
#pragma unroll
            for (int u = 0; u < AU; ++u) {
                const int unit = tid + u * TC5_PRODUCERS, i = unit % TC5_BM, c = unit / TC5_BM;
                uint4 rh, rl, ih, il;
                split4(av[u], rh, rl, ih, il);
                const size_t off = (size_t)c * TC5_BM * 16 + (size_t)i * 16;
                *reinterpret_cast<uint4*>(st + off) = rh;
                *reinterpret_cast<uint4*>(st + Cfg::A_PART + off) = rl;
                *reinterpret_cast<uint4*>(st + 2 * Cfg::A_PART + off) = ih;
                *reinterpret_cast<uint4*>(st + 3 * Cfg::A_PART + off) = il;
            }
#pragma unroll
            for (int u = 0; u < BU; ++u) {
                const int unit = tid + u * TC5_PRODUCERS, j = unit / 4, c = unit % 4;
                if (unit >= BT) continue;
                uint4 rh, rl, ih, il;
                split4(bv[u], rh, rl, ih, il);
                const size_t off = (size_t)c * BN * 16 + (size_t)j * 16;
                *reinterpret_cast<uint4*>(sb + off) = rh;
                *reinterpret_cast<uint4*>(sb + Cfg::B_PART + off) = rl;
                *reinterpret_cast<uint4*>(sb + 2 * Cfg::B_PART + off) = ih;
                *reinterpret_cast<uint4*>(sb + 3 * Cfg::B_PART + off) = il;
            }
        };
        constexpr int AHEAD = Cfg::AHEAD;
        // prologue: the first AHEAD k-blocks into fresh stages, one commit group each
        for (int q = 0; q < AHEAD; ++q) {
            if (q < nkb) issue(q, q);
            cp_async_commit();
        }
        bool ok = true;
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % STAGES;
            // groups committed so far: AHEAD + kb; k-block kb is the (kb+1)-th
            cp_async_wait<AHEAD - 1>();
            producers_sync();                    // every producer's copies of stage s have landed
            convert(s);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic -> async proxy
            mbar_arrive(full0 + 8 * s);
            const int kn = kb + AHEAD;
            if (kn < nkb) {
                const int sn = kn % STAGES;
                if (kn >= STAGES) {
                    // the MMAs of k-block kn - STAGES (= kb - 1) read stage sn: one thread waits
                    // (bounded), the others at the barrier, which also agrees on giving up
                    bool bad = false;
                    if (tid == 0) bad = !mbar_wait(empty0 + 8 * sn, (uint32_t)(((kn / STAGES) - 1) & 1), &abort_flag);
                    if (producers_any(bad || abort_flag)) {
                        ok = false;
                        break;
                    }
                }
                issue(kn, sn);
            }
            cp_async_commit();
        }
        cp_async_wait<0>();                      // no copy may still target this CTA's memory
        if (!ok) {
            abort_flag = 1;
            atomicOr(status, RB_TC5_TIMEOUT);
        }
        // ---------------- epilogue ------------------------------------------------------------------
        // warp-uniform: the accumulator reads below are warp-collective
        const bool done = __all_sync(0xffffffffu, mbar_wait(done_bar, 0u, &abort_flag) && !abort_flag);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!done) {
            if (lane == 0 && !abort_flag) atomicOr(status, RB_TC5_TIMEOUT);
        } else {
            const int quarter = warp & 3, half = warp >> 2;
            const int row = quarter * 32 + lane;
            const int gi = m0 + row;
            const bool live = gi < m;
            long long dro = 0, cro = 0;
            bool use_c = false;
            if (live) {
                dro = vrow(sd.D, gi);
                use_c = sd.C.p && !(gi >= sd.nobeta_r0 && gi < sd.nobeta_r1);
                if (use_c) cro = vrow(sd.C, gi);
            }
            const z alpha = sd.alpha, beta = sd.beta;
            z* pp = part ? part + ((long long)blockIdx.y * ksplit + blockIdx.z) * pstride : nullptr;
            constexpr int HALF = BN / 2;
            constexpr int CH = HALF < 16 ? HALF : 16;
#pragma unroll 1
            for (int c0 = half * HALF; c0 < (half + 1) * HALF; c0 += CH) {
                float vr[16], vi[16];
                const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
                tmem_ld16(tmem + lane_base + (uint32_t)c0, vr);
                tmem_ld16(tmem + lane_base + (uint32_t)(BN + c0), vi);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (!live) continue;
#pragma unroll
                for (int e = 0; e < CH; ++e) {
                    const int gj = n0 + c0 + e;
                    if (gj >= n) break;
                    if (pp) {
                        pp[gi + (long long)gj * ldp] = zmk((double)vr[e], (double)vi[e]);
                        continue;
                    }
                    z v = zmul(alpha, zmk((double)vr[e], (double)vi[e]));
                    if (use_c) zfma(v, beta, sd.C.p[cro + (long long)vcol(sd.C, gj) * sd.C.ld]);
                    sd.D.p[dro + (long long)vcol(sd.D, gj) * sd.D.ld] = v;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 8) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)Cfg::TMEM_COLS));
    }
}

template <int BN>
static cudaError_t launch_tc5(const GemmBatch& b, int* status, cudaStream_t s) {
    using Cfg = Tc5Cfg<BN>;
    static DeviceAttrCache attr;
    cudaError_t e = ensure_smem_attr(zgemm_tc5_kernel<BN>, Cfg::SMEM, attr, true);
    if (e != cudaSuccess) return e;
    const int tiles = ((b.max_m + TC5_BM - 1) / TC5_BM) * ((b.max_n + BN - 1) / BN);
    if (b.t5_ksplit > 1 && b.work) {
        if (b.count > 65535 || b.t5_ksplit > 65535) return cudaErrorInvalidValue;
        zgemm_tc5_kernel<BN><<<dim3(tiles, b.count, b.t5_ksplit), TC5_THREADS, Cfg::SMEM, s>>>(
            b.d_desc, status, b.t5_kchunk, b.work, b.t5_pstride, b.max_m, b.t5_ksplit);
        note_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        return launch_gemm_reduce(b, b.t5_ksplit, b.t5_pstride, s);
    }
    for (int off = 0; off < b.count; off += 65535) {
        const int cnt = (b.count - off) < 65535 ? (b.count - off) : 65535;
        zgemm_tc5_kernel<BN><<<dim3(tiles, cnt), TC5_THREADS, Cfg::SMEM, s>>>(b.d_desc + off, status, 0, nullptr, 0,
                                                                             0, 1);
        note_launch();
    }
    return cudaGetLastError();
}

long long gemm_plan_split_tc5_factor(GemmBatch& b) {
    b.t5_ksplit = 1;
    b.t5_kchunk = 0;
    b.t5_pstride = 0;
    // the factor's stages of the middle levels (a few nodes, m = 256 .. 512) give too few 128-row
    // tiles for 148 SMs: split k until about 1.5 waves, each range at least 128 deep.  Stages
    // that fill a wave already are left whole (their outputs are large: a reduction pass would
    // cost more than it gains).
    if (b.count == 0 || b.max_k < 256) return 0;
    const int bn = tc5_tile_n(b);
    const long long tiles =
        (long long)b.count * ((b.max_m + TC5_BM - 1) / TC5_BM) * ((b.max_n + bn - 1) / bn);
    if (tiles >= 148) return 0;
    long long sp = (222 + tiles - 1) / tiles;
    sp = std::min<long long>(sp, 8);
    sp = std::min<long long>(sp, b.max_k / 128);
    if (sp < 2) return 0;
    const int kc = (int)(((b.max_k + sp - 1) / sp + TC5_KB - 1) / TC5_KB * TC5_KB);
    const int ks = (b.max_k + kc - 1) / kc;
    if (ks < 2) return 0;
    b.t5_kchunk = kc;
    b.t5_ksplit = ks;
    b.t5_pstride = (long long)b.max_m * b.max_n;
    return (long long)b.count * ks * b.t5_pstride;
}

long long gemm_plan_split_tc5(GemmBatch& b) {
    b.t5_ksplit = 1;
    b.t5_kchunk = 0;
    b.t5_pstride = 0;
    if (b.count == 0 || b.max_k < 128) return 0;
    // about two waves of one CTA per SM from the 128-row tiles alone (n-independent), each range
    // at least 64 deep
    const long long ctas = (long long)b.count * ((b.max_m + TC5_BM - 1) / TC5_BM);
    long long sp = (2 * 148 + ctas - 1) / ctas;
    sp = std::min<long long>(sp, 32);
    sp = std::min<long long>(sp, b.max_k / 64);
    if (sp < 2) return 0;
    const int kc = (int)(((b.max_k + sp - 1) / sp + TC5_KB - 1) / TC5_KB * TC5_KB);
    const int ks = (b.max_k + kc - 1) / kc;
    if (ks < 2) return 0;
    b.t5_kchunk = kc;
    b.t5_ksplit = ks;
    b.t5_pstride = (long long)b.max_m * b.max_n;
    return (long long)b.count * ks * b.t5_pstride;
}

int tc5_tile_n(const GemmBatch& b) {
    // n columns per tile: 32 for the narrow solve products, 128 where the 128 x 128 tiles still
    // fill a wave of the 148 SMs (twice the operand reuse of 128 x 64), else 64
    if (b.max_n <= 32) return 32;
    if (b.max_n <= 64) return 64;
    const long long t128 = (long long)b.count * ((b.max_m + TC5_BM - 1) / TC5_BM) * ((b.max_n + 127) / 128);
    return t128 >= 148 ? 128 : 64;
}

cudaError_t launch_gemm_tc5(const GemmBatch& b, int* status, cudaStream_t s) {
    if (b.count == 0 || b.max_m == 0 || b.max_n == 0) return cudaSuccess;
    if (!status) return cudaErrorInvalidValue;
    const int bn = tc5_tile_n(b);
    if (bn == 32) return launch_tc5<32>(b, status, s);
    if (bn == 128) return launch_tc5<128>(b, status, s);
    return launch_tc5<64>(b, status, s);
}

}  // namespace rb
