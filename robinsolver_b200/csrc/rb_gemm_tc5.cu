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
// Two kernels per batch:
//  1. tc5_split_kernel converts every operand element ONCE: it reads the FP64 operands through
//     the problems' ZViews (face gathers, row maps, skipped bands, exactly as the FP64 kernels
//     read them), splits each value into TF32 hi/lo with integer operations on the FP64 bit
//     pattern (the FP64 -> FP32 conversion instructions run on the narrow XU pipe, which bounded
//     a kernel that converted inside the GEMM once per output tile), and writes "planes": per
//     problem, per 128-row (A) or BN-column (B) tile and per 16-deep k-block one contiguous block
//     laid out exactly as the GEMM's shared-memory stage holds it (the UMMA K-major no-swizzle
//     layout: 16-byte rows of four K values, 128-byte core matrices of 8 rows), zero outside the
//     problem.
//  2. zgemm_tc5_kernel, one CTA per 128 x BN output tile, 8 warps:
//       warp 0   one lane streams the k-blocks of A and B into a ring of shared-memory stages with
//                two 1-D bulk copies each (cp.async.bulk, completion counted in bytes on the
//                stage's mbarrier; each CTA copies only for itself);
//       warp 1   allocates 2*BN tensor-memory columns; one lane issues the stage's MMAs once its
//                bytes have landed and releases the stage with tcgen05.commit;
//       all 8   the epilogue: tcgen05.ld of the accumulators (warp w reads lanes 32 (w % 4) ..
//                +31, half w / 4 of the columns), alpha/beta, scatter through the output maps.
// Every mbarrier wait is bounded (RB_TC5_WAIT_NS on the global timer).  A wait that runs out sets
// RB_TC5_TIMEOUT in the status word, the CTA stops issuing work, waits (bounded) for the copies
// and MMAs it issued, frees its tensor memory and returns.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "rb_kernels.h"

namespace rb {

namespace {

constexpr int TC5_BM = 128;          // output rows per tile = UMMA M (one lane per row)
constexpr int TC5_KB = 16;           // complex k per block / stage: 4 chunks of 4 TF32 = two UMMA k-steps
constexpr int TC5_THREADS = 256;     // 8 warps
constexpr int TC5_A_BLOCK = TC5_BM * TC5_KB * 16;          // bytes of one A plane block (32 KB)
constexpr unsigned long long RB_TC5_WAIT_NS = 1000000000ull;   // 1 s per wait

template <int BN>
struct Tc5Cfg {
    static constexpr int A_PART = TC5_BM * TC5_KB * 4;     // one TF32 part of an A block
    static constexpr int B_BLOCK = BN * TC5_KB * 16;       // bytes of one B plane block
    static constexpr int B_PART = BN * TC5_KB * 4;
    static constexpr int STAGE = TC5_A_BLOCK + B_BLOCK;
    static constexpr int STAGES = (204800 / STAGE) < 4 ? (204800 / STAGE) : 4;   // 4, 4, 3, 2 for BN 32..256
    static constexpr int SMEM = STAGES * STAGE + 1024;     // + 1024 for the alignment of the stages
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

// one arrival that also announces `bytes` of bulk-copy data the phase must wait for
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
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
// another warp has already given up (*abort, if given)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned it = 0;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 63) == 63) {
            if (abort && *abort) return false;
            if (global_ns() - t0 > RB_TC5_WAIT_NS) return false;
        }
    }
}

// 1-D bulk copy global -> this CTA's shared memory, completion counted on an mbarrier
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
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

// TF32 bit pattern (an FP32 pattern whose low 13 mantissa bits are zero) of a double given by
// its high word, rounded already to 10 mantissa bits (the low 10 bits of hw and the low word
// are zero).  Below the FP32 normal range: signed zero; above it (and inf/NaN): signed infinity.
__device__ __forceinline__ uint32_t tf32_of_rounded_hiword(uint32_t hw) {
    const uint32_t e = (hw >> 20) & 0x7FFu;
    const uint32_t sign = hw & 0x80000000u;
    if (e <= 896u) return sign;
    if (e >= 1151u) return sign | 0x7F800000u;
    // ((e - 896) << 23) | (top 10 mantissa bits << 13): the exponent rebiased from 1023 to 127
    return sign | (((hw & 0x7FFFFFFFu) - (896u << 20)) << 3);
}

// x -> (hi, lo) TF32 patterns: hi = x rounded to 11 significant bits (to nearest, ties away
// from zero), lo = (x - hi) rounded the same way; x - hi is exact in FP64.  Integer operations
// and one FP64 subtraction only.
__device__ __forceinline__ void split_tf32(double x, uint32_t& hi, uint32_t& lo) {
    const uint32_t hr = ((uint32_t)__double2hiint(x) + 0x200u) & 0xFFFFFC00u;
    hi = tf32_of_rounded_hiword(hr);
    const double r = x - __hiloint2double((int)hr, 0);
    lo = tf32_of_rounded_hiword(((uint32_t)__double2hiint(r) + 0x200u) & 0xFFFFFC00u);
}

// Operand plane geometry of a batch: MT 128-row tiles of A, NT BN-column tiles of B, KBN
// 16-deep k-blocks; A blocks first ([problem][mt][kb]), then B blocks ([problem][nt][kb]).
struct PlaneGeom {
    int MT, NT, KBN;
    long long a_bytes;     // all A blocks
};
PlaneGeom plane_geom(const GemmBatch& b, int bn) {
    PlaneGeom g;
    g.MT = (b.max_m + TC5_BM - 1) / TC5_BM;
    g.NT = (b.max_n + bn - 1) / bn;
    g.KBN = (b.max_k + TC5_KB - 1) / TC5_KB;
    g.a_bytes = (long long)b.count * g.MT * g.KBN * TC5_A_BLOCK;
    return g;
}

}  // namespace

// One CTA converts one slab: 128 rows of an A block (row i of A = output row), or up to 128
// columns of a B block (column j of B = output column), 16 k deep.  Slab s < nA: A slab
// (problem, mt, kb); else B slab (problem, nt, kb, half) with BN / min(BN, 128) slabs per block.
template <int BN>
__global__ void __launch_bounds__(256) tc5_split_kernel(const GemmDesc* __restrict__ descs, int MT, int NT, int KBN,
                                                        long long nA, unsigned char* __restrict__ planes,
                                                        long long a_bytes) {
    constexpr int BR = BN < 128 ? BN : 128;           // rows of a B slab
    constexpr int BSLABS = BN / BR;                   // slabs per B block
    __shared__ z S[128][TC5_KB + 1];                  // [row][k], padded against bank conflicts
    const int tid = threadIdx.x;
    long long s = blockIdx.x;
    const bool isA = s < nA;
    int prob, tile, kb, half = 0;
    if (isA) {
        kb = (int)(s % KBN);
        s /= KBN;
        tile = (int)(s % MT);
        prob = (int)(s / MT);
    } else {
        s -= nA;
        half = (int)(s % BSLABS);
        s /= BSLABS;
        kb = (int)(s % KBN);
        s /= KBN;
        tile = (int)(s % NT);
        prob = (int)(s / NT);
    }
    const GemmDesc& g = descs[prob];
    const int k0 = kb * TC5_KB;
    const int R = isA ? 128 : BR;
    const int r0 = isA ? tile * TC5_BM : tile * BN + half * BR;     // first row (A) / column (B)
    if (isA) {
        // consecutive threads take consecutive rows of one column of A (column-major)
        const ZView v = g.A;
        for (int e = tid; e < 128 * TC5_KB; e += 256) {
            const int r = e % 128, kk = e / 128, i = r0 + r, k = k0 + kk;
            z val = zmk(0.0, 0.0);
            if (i < g.m && k < g.k) val = v.p[vrow(v, i) + (long long)vcol(v, k) * v.ld];
            S[r][kk] = val;
        }
    } else {
        // consecutive threads take consecutive k of one column of B
        const ZView v = g.B;
        for (int e = tid; e < BR * TC5_KB; e += 256) {
            const int kk = e % TC5_KB, r = e / TC5_KB, j = r0 + r, k = k0 + kk;
            z val = zmk(0.0, 0.0);
            if (j < g.n && k < g.k) val = v.p[vrow(v, k) + (long long)vcol(v, j) * v.ld];
            S[r][kk] = val;
        }
    }
    __syncthreads();
    // unit (row r, K chunk c): four k values -> four 16-byte TF32 parts at
    // block + ((part * 4 + c) * ROWS + row) * 16
    const int ROWS = isA ? TC5_BM : BN;
    unsigned char* blk = isA ? planes + (((long long)prob * MT + tile) * KBN + kb) * TC5_A_BLOCK
                             : planes + a_bytes + (((long long)prob * NT + tile) * KBN + kb) * (long long)(BN * TC5_KB * 16);
    const int rofs = isA ? 0 : half * BR;
    for (int u = tid; u < R * 4; u += 256) {
        const int r = u % R, c = u / R;
        uint4 rh, rl, ih, il;
        split_tf32(S[r][4 * c + 0].x, rh.x, rl.x); split_tf32(S[r][4 * c + 0].y, ih.x, il.x);
        split_tf32(S[r][4 * c + 1].x, rh.y, rl.y); split_tf32(S[r][4 * c + 1].y, ih.y, il.y);
        split_tf32(S[r][4 * c + 2].x, rh.z, rl.z); split_tf32(S[r][4 * c + 2].y, ih.z, il.z);
        split_tf32(S[r][4 * c + 3].x, rh.w, rl.w); split_tf32(S[r][4 * c + 3].y, ih.w, il.w);
        const long long row = rofs + r;
        uint4* o = reinterpret_cast<uint4*>(blk);
        o[(0 * 4 + c) * (long long)ROWS + row] = rh;
        o[(1 * 4 + c) * (long long)ROWS + row] = rl;
        o[(2 * 4 + c) * (long long)ROWS + row] = ih;
        o[(3 * 4 + c) * (long long)ROWS + row] = il;
    }
}

// Split-K (part != nullptr): blockIdx.z takes k in [z * kchunk, (z + 1) * kchunk) (kchunk a
// multiple of 16) and writes its raw sums to part + (problem * ksplit + z) * pstride + i + j * ldp;
// the reduction kernel finishes.  prob0: index of descs[0] in the batch (the planes are indexed
// by the batch's problem index).
template <int BN>
__global__ void __launch_bounds__(TC5_THREADS, 1) zgemm_tc5_kernel(const GemmDesc* __restrict__ descs, int prob0,
                                                                  int* status, const unsigned char* __restrict__ planes,
                                                                  int MT, int NT, int KBN, long long a_bytes,
                                                                  int kchunk, z* part, long long pstride, int ldp,
                                                                  int ksplit) {
    using Cfg = Tc5Cfg<BN>;
    constexpr int STAGES = Cfg::STAGES;
    extern __shared__ __align__(1024) unsigned char tc5_smem[];
    __shared__ GemmDesc sd;
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
    const int tm = blockIdx.x % tiles_m, tn = blockIdx.x / tiles_m;
    const int m0 = tm * TC5_BM;
    const int n0 = tn * BN;
    const int kb0 = kbeg / TC5_KB;
    const int nkb = (K - kbeg + TC5_KB - 1) / TC5_KB;
    const long long prob = prob0 + (long long)blockIdx.y;
    const unsigned char* gA = planes + ((prob * MT + tm) * KBN + kb0) * (long long)TC5_A_BLOCK;
    const unsigned char* gB = planes + a_bytes + ((prob * NT + tn) * KBN + kb0) * (long long)Cfg::B_BLOCK;

    unsigned char* stage_base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(tc5_smem) + 1023) & ~uintptr_t(1023));
    const uint32_t full0 = smem_u32(&bars[0]);
    const uint32_t empty0 = smem_u32(&bars[STAGES]);
    const uint32_t done_bar = smem_u32(&bars[2 * STAGES]);

    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"((uint32_t)Cfg::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    if (warp == 0) {
        // ---------------- producer: one lane, the warp kept converged --------------------------------
        bool ok = true;
        int issued = 0;
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % STAGES;
            if (kb >= STAGES) {
                // the MMAs of k-block kb - STAGES read stage s
                ok = __all_sync(0xffffffffu, mbar_wait(empty0 + 8 * s, (uint32_t)(((kb / STAGES) - 1) & 1), &abort_flag));
                if (!ok) break;
            }
            if (lane == 0) {
                const uint32_t st = smem_u32(stage_base + (size_t)s * Cfg::STAGE);
                mbar_arrive_expect_tx(full0 + 8 * s, (uint32_t)Cfg::STAGE);
                bulk_g2s(st, gA + (long long)kb * TC5_A_BLOCK, (uint32_t)TC5_A_BLOCK, full0 + 8 * s);
                bulk_g2s(st + TC5_A_BLOCK, gB + (long long)kb * Cfg::B_BLOCK, (uint32_t)Cfg::B_BLOCK, full0 + 8 * s);
            }
            __syncwarp();
            issued = kb + 1;
        }
        if (!ok) {
            abort_flag = 1;
            if (lane == 0) atomicOr(status, RB_TC5_TIMEOUT);
            // no copy may still target this CTA's memory when it exits: wait (bounded) for the
            // stages filled last, whatever the MMA warp did with them
            for (int kb = max(0, issued - STAGES); kb < issued; ++kb)
                mbar_wait(full0 + 8 * (kb % STAGES), (uint32_t)((kb / STAGES) & 1), nullptr);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------- MMA issuer: one lane, the warp kept converged ----------------------------
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
                const uint32_t bb = st + TC5_A_BLOCK;
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
    }

    // ---------------- epilogue: all 8 warps ----------------------------------------------------------
    // warp-uniform: the accumulator reads below are warp-collective
    const bool done = __all_sync(0xffffffffu, mbar_wait(done_bar, 0u, nullptr) && !abort_flag);
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
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
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
    const PlaneGeom pg = plane_geom(b, BN);
    unsigned char* planes = static_cast<unsigned char*>(b.t5_planes);
    // 1. the operand planes: every A slab, then every B slab
    {
        constexpr int BSLABS = BN / (BN < 128 ? BN : 128);
        const long long nA = (long long)b.count * pg.MT * pg.KBN;
        const long long nB = (long long)b.count * pg.NT * pg.KBN * BSLABS;
        if (nA + nB > 0x7FFFFFFFLL) return cudaErrorInvalidValue;
        tc5_split_kernel<BN><<<(unsigned)(nA + nB), 256, 0, s>>>(b.d_desc, pg.MT, pg.NT, pg.KBN, nA, planes,
                                                                 pg.a_bytes);
        note_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    // 2. the products
    const int tiles = ((b.max_m + TC5_BM - 1) / TC5_BM) * ((b.max_n + BN - 1) / BN);
    if (b.t5_ksplit > 1 && b.work) {
        if (b.count > 65535 || b.t5_ksplit > 65535 || b.t5_kchunk % TC5_KB) return cudaErrorInvalidValue;
        zgemm_tc5_kernel<BN><<<dim3(tiles, b.count, b.t5_ksplit), TC5_THREADS, Cfg::SMEM, s>>>(
            b.d_desc, 0, status, planes, pg.MT, pg.NT, pg.KBN, pg.a_bytes, b.t5_kchunk, b.work, b.t5_pstride,
            b.max_m, b.t5_ksplit);
        note_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        return launch_gemm_reduce(b, b.t5_ksplit, b.t5_pstride, s);
    }
    for (int off = 0; off < b.count; off += 65535) {
        const int cnt = (b.count - off) < 65535 ? (b.count - off) : 65535;
        zgemm_tc5_kernel<BN><<<dim3(tiles, cnt), TC5_THREADS, Cfg::SMEM, s>>>(
            b.d_desc + off, off, status, planes, pg.MT, pg.NT, pg.KBN, pg.a_bytes, 0, nullptr, 0, 0, 1);
        note_launch();
    }
    return cudaGetLastError();
}

// ================= int8 digit-slice engine (Ozaki scheme) =====================================
//
// Every row of A (and column of B) is scaled by a power of two 2^-e so that its largest component
// (re or im) is below 1/2, and each scaled value v is written as OZ_S balanced base-128 digits,
// v = sum_j d_j 128^-j + r with d_j in [-64, 64] and |r| <= 2^(-7 OZ_S - 1).  A real product is
// then sum_{j,j'} d_j d'_j' 128^-(j+j') 2^(e+f); the digit products of one diagonal j + j' = t share
// that weight, so they accumulate EXACTLY in one int32 tensor-memory accumulator (|d d'| <= 4096,
// at most 2 (t - 1) products per k: no overflow below k = 32768).  Pairs with j + j' > OZ_S + 1 are
// dropped.  The epilogue combines the OZ_S diagonals in FP64 with their weights and the row and
// column scales.  Normwise error about 2^-35 of max|A_i.| max|B_.j| k, against ~1e-7 for split
// TF32 with FP32 accumulation, for 60 int8 MMAs per complex k-step of 32 (int8 runs at four times
// the TF32 rate: about the tensor work of TF32x3).
// Complex: Cr = Ar Br + Ai (-Bi), Ci = Ar Bi + Ai Br (int8 MMAs have no negate bit, so -Bi has its
// own digits).  A digit plane of B holds 144 rows, [-Bi | Br | Bi] (48 columns each), so one MMA of
// N = 96 takes Ar against rows 48..143 ([Br | Bi]) and one takes Ai against rows 0..95 ([-Bi | Br]):
// the accumulator of diagonal t (columns (t - 2) * 96 ..) holds Cr in its first 48 columns and Ci in
// the next 48.  Two MMAs per digit pair, 30 per k-block.
constexpr int OZ_S = 5;                                    // digits per value
constexpr int OZ_KB = 32;                                  // k per block / stage = one int8 MMA K
constexpr int OZ_BN = 48;                                  // OZ_S accumulators x (48 re + 48 im) columns <= 512
constexpr int OZ_MMA_N = 2 * OZ_BN;
constexpr int OZ_B_ROWS = 3 * OZ_BN;                       // -Bi | Br | Bi
constexpr int OZ_A_PLANES = 2 * OZ_S;                      // Ar, Ai digits
constexpr int OZ_B_PLANES = OZ_S;                          // [-Bi | Br | Bi] digits
constexpr int OZ_A_PLANE = 2 * TC5_BM * 16;                // one digit plane of an A block: 2 K chunks x 128 rows x 16 B
constexpr int OZ_B_PLANE = 2 * OZ_B_ROWS * 16;
constexpr int OZ_A_BLOCK = OZ_A_PLANES * OZ_A_PLANE;       // 40960
constexpr int OZ_B_BLOCK = OZ_B_PLANES * OZ_B_PLANE;       // 23040
constexpr int OZ_STAGE = OZ_A_BLOCK + OZ_B_BLOCK;
constexpr int OZ_STAGES = 3;
constexpr int OZ_SMEM = OZ_STAGES * OZ_STAGE + 1024;
constexpr int OZ_TMEM_COLS = 512;
constexpr int OZ_MAX_K = 32768;                            // int32 accumulators stay exact below this k
static_assert(OZ_BN % 8 == 0, "the column-scale kernel runs whole warps of 8 columns per block");

namespace {

// frexp exponent of |x| (x = m 2^ex, m in [0.5, 1)); -1022 for zero and subnormals
__device__ __forceinline__ int oz_exponent(double x) {
    return (int)(((uint32_t)__double2hiint(x) >> 20) & 0x7FFu) - 1022;
}

// exact 2^p for -1022 <= p <= 1023
__device__ __forceinline__ double oz_pow2(int p) {
    return __hiloint2double((p + 1023) << 20, 0);
}

// OZ_S balanced base-128 digits of v, |v| < 1/2: round(128 v) by the 1.5 * 2^52 rounding constant
// (its low word holds the integer), the exact remainder carried to the next digit
__device__ __forceinline__ void oz_digits(double v, int (&d)[OZ_S]) {
    const double magic = 6755399441055744.0;
#pragma unroll
    for (int j = 0; j < OZ_S; ++j) {
        const double y = v * 128.0;
        const double t = __dadd_rn(y, magic);
        d[j] = __double2loint(t);
        v = __dadd_rn(y, -__dadd_rn(t, -magic));
    }
}

// Operand plane geometry of a batch on the int8 engine: MT 128-row tiles of A, NT 48-column tiles
// of B, KBN 32-deep k-blocks; A blocks ([problem][mt][kb]), B blocks ([problem][nt][kb]), then the
// row exponents of A ([problem][MT * 128]) and the column exponents of B ([problem][NT * 48]).
struct OzGeom {
    int MT, NT, KBN;
    long long a_bytes, b_bytes, ea_off, fb_off, total;
};
OzGeom oz_geom(const GemmBatch& b) {
    OzGeom g;
    g.MT = (b.max_m + TC5_BM - 1) / TC5_BM;
    g.NT = (b.max_n + OZ_BN - 1) / OZ_BN;
    g.KBN = (b.max_k + OZ_KB - 1) / OZ_KB;
    g.a_bytes = (long long)b.count * g.MT * g.KBN * OZ_A_BLOCK;
    g.b_bytes = (long long)b.count * g.NT * g.KBN * OZ_B_BLOCK;
    g.ea_off = g.a_bytes + g.b_bytes;
    g.fb_off = g.ea_off + 4LL * b.count * g.MT * TC5_BM;
    g.total = (g.fb_off + 4LL * b.count * g.NT * OZ_BN + 255) / 256 * 256;
    return g;
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int (&v)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}

// instruction descriptor of kind::i8: D S32, A and B signed 8-bit, both K-major, M = 128, N = 96
__host__ __device__ constexpr uint32_t oz_idesc() {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OZ_MMA_N >> 3) << 17) | ((uint32_t)(TC5_BM >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

}  // namespace

// Row exponents of A: e = 1 + max frexp exponent over the row's k (re and im), so the scaled row
// lies in (-1/2, 1/2).  Block = 32 rows x 8 k phases over one range of OZ_SCALE_KC k (blockIdx.y);
// grid = (count * ceil(MT * 128 / 32), ceil(max_k / OZ_SCALE_KC)).  The ranges meet in an atomic
// max on ea, which the launcher fills with INT_MIN-like bytes first (a whole row per block left
// most SMs idle, waiting on one long chain of loads each).
constexpr int OZ_SCALE_KC = 64;
__global__ void __launch_bounds__(256) oz_scale_a_kernel(const GemmDesc* __restrict__ descs, int MT, int* ea) {
    __shared__ int red[8][32];
    const int groups = MT * TC5_BM / 32;
    const int prob = blockIdx.x / groups, grp = blockIdx.x % groups;
    const int lane = threadIdx.x & 31, ph = threadIdx.x >> 5;
    const GemmDesc& g = descs[prob];
    const int i = grp * 32 + lane;
    const int k0 = blockIdx.y * OZ_SCALE_KC, k1 = min(g.k, k0 + OZ_SCALE_KC);
    if (k0 >= g.k && blockIdx.y > 0) return;          // uniform over the block
    int ex = -1022;
    if (i < g.m) {
        const ZView v = g.A;
        const long long ro = vrow(v, i);
#pragma unroll 4
        for (int k = k0 + ph; k < k1; k += 8) {
            const z x = v.p[ro + (long long)vcol(v, k) * v.ld];
            ex = max(ex, max(oz_exponent(x.x), oz_exponent(x.y)));
        }
    }
    red[ph][lane] = ex;
    __syncthreads();
    if (ph == 0) {
#pragma unroll
        for (int q = 1; q < 8; ++q) ex = max(ex, red[q][lane]);
        atomicMax(ea + (long long)prob * MT * TC5_BM + i, ex + 1);
    }
}

// Column exponents of B, one warp per column (k runs contiguously down a column of B's view).
__global__ void __launch_bounds__(256) oz_scale_b_kernel(const GemmDesc* __restrict__ descs, int NT, int* fb) {
    const int cols = NT * OZ_BN;
    const long long w = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const int prob = (int)(w / cols), j = (int)(w % cols);
    const GemmDesc& g = descs[prob];
    int ex = -1022;
    if (j < g.n) {
        const ZView v = g.B;
        const long long co = (long long)vcol(v, j) * v.ld;
        for (int k = lane; k < g.k; k += 32) {
            const z x = v.p[vrow(v, k) + co];
            ex = max(ex, max(oz_exponent(x.x), oz_exponent(x.y)));
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) ex = max(ex, __shfl_xor_sync(0xffffffffu, ex, o));
    if (lane == 0) fb[(long long)prob * cols + j] = ex + 1;
}

// Digit planes of one slab: s < nA an A block (problem, mt, kb: 128 rows x 32 k, in two 16-k
// halves), else a B block (problem, nt, kb: 48 columns x 32 k).  Digit plane p of a block holds
// chunk c (16 k) of row r at ((p * 2 + c) * ROWS + r) * 16 bytes; a B plane's rows are -Bi of the
// 48 columns, then Br, then Bi.
__global__ void __launch_bounds__(256, 4) oz_split_kernel(const GemmDesc* __restrict__ descs, int MT, int NT, int KBN,
                                                       long long nA, unsigned char* __restrict__ planes,
                                                       long long a_bytes, const int* __restrict__ ea,
                                                       const int* __restrict__ fb) {
    __shared__ z S[128 * 17];
    const int tid = threadIdx.x;
    long long s = blockIdx.x;
    const bool isA = s < nA;
    if (!isA) s -= nA;
    const int kb = (int)(s % KBN);
    s /= KBN;
    const int tiles = isA ? MT : NT;
    const int tile = (int)(s % tiles);
    const int prob = (int)(s / tiles);
    const GemmDesc& g = descs[prob];
    if (isA) {
        unsigned char* blk = planes + (((long long)prob * MT + tile) * KBN + kb) * OZ_A_BLOCK;
        const ZView v = g.A;
        for (int half = 0; half < 2; ++half) {
            const int k0 = kb * OZ_KB + half * 16;
            for (int e = tid; e < 128 * 16; e += 256) {
                const int r = e % 128, kk = e / 128, i = tile * TC5_BM + r, k = k0 + kk;
                z val = zmk(0.0, 0.0);
                if (i < g.m && k < g.k) val = v.p[vrow(v, i) + (long long)vcol(v, k) * v.ld];
                S[r * 17 + kk] = val;
            }
            __syncthreads();
            {
                // unit: row r, part (0 re, 1 im): 16 values -> OZ_S digit chunks of 16 bytes
                const int r = tid % 128, part = tid / 128;
                const double sc = oz_pow2(-ea[((long long)prob * MT + tile) * TC5_BM + r]);
                uint32_t w[OZ_S][4];
#pragma unroll
                for (int j = 0; j < OZ_S; ++j) w[j][0] = w[j][1] = w[j][2] = w[j][3] = 0u;
#pragma unroll
                for (int kk = 0; kk < 16; ++kk) {
                    const z x = S[r * 17 + kk];
                    int d[OZ_S];
                    oz_digits((part ? x.y : x.x) * sc, d);
#pragma unroll
                    for (int j = 0; j < OZ_S; ++j) w[j][kk >> 2] |= ((uint32_t)d[j] & 0xFFu) << (8 * (kk & 3));
                }
#pragma unroll
                for (int j = 0; j < OZ_S; ++j) {
                    const int p = part * OZ_S + j;
                    *reinterpret_cast<uint4*>(blk + ((long long)(p * 2 + half) * TC5_BM + r) * 16) =
                        make_uint4(w[j][0], w[j][1], w[j][2], w[j][3]);
                }
            }
            __syncthreads();
        }
    } else {
        unsigned char* blk = planes + a_bytes + (((long long)prob * NT + tile) * KBN + kb) * OZ_B_BLOCK;
        const ZView v = g.B;
        const int k0 = kb * OZ_KB;
        for (int e = tid; e < OZ_BN * OZ_KB; e += 256) {
            const int kk = e % OZ_KB, c = e / OZ_KB, j = tile * OZ_BN + c, k = k0 + kk;
            z val = zmk(0.0, 0.0);
            if (j < g.n && k < g.k) val = v.p[vrow(v, k) + (long long)vcol(v, j) * v.ld];
            S[c * 33 + kk] = val;
        }
        __syncthreads();
        if (tid < OZ_BN * 4) {
            // unit: column c, part (0 re, 1 im), half (16 k)
            const int c = tid % OZ_BN, part = (tid / OZ_BN) & 1, half = tid / (2 * OZ_BN);
            const double sc = oz_pow2(-fb[((long long)prob * NT + tile) * OZ_BN + c]);
            uint32_t w[OZ_S][4], wn[OZ_S][4];
#pragma unroll
            for (int j = 0; j < OZ_S; ++j)
                w[j][0] = w[j][1] = w[j][2] = w[j][3] = wn[j][0] = wn[j][1] = wn[j][2] = wn[j][3] = 0u;
#pragma unroll
            for (int kk = 0; kk < 16; ++kk) {
                const z x = S[c * 33 + half * 16 + kk];
                int d[OZ_S];
                oz_digits((part ? x.y : x.x) * sc, d);
#pragma unroll
                for (int j = 0; j < OZ_S; ++j) {
                    w[j][kk >> 2] |= ((uint32_t)d[j] & 0xFFu) << (8 * (kk & 3));
                    wn[j][kk >> 2] |= ((uint32_t)(-d[j]) & 0xFFu) << (8 * (kk & 3));
                }
            }
#pragma unroll
            for (int j = 0; j < OZ_S; ++j) {
                unsigned char* pl = blk + (long long)(j * 2 + half) * OZ_B_ROWS * 16;
                // Br at rows 48.., Bi at rows 96.. and -Bi at rows 0..
                *reinterpret_cast<uint4*>(pl + (long long)((part ? 2 : 1) * OZ_BN + c) * 16) =
                    make_uint4(w[j][0], w[j][1], w[j][2], w[j][3]);
                if (part)
                    *reinterpret_cast<uint4*>(pl + (long long)c * 16) = make_uint4(wn[j][0], wn[j][1], wn[j][2], wn[j][3]);
            }
        }
    }
}

// One CTA per 128 x 48 output tile, 8 warps, the TF32x3 kernel's roles and bounded waits; per
// stage (k-block of 32) 15 digit pairs x 2 MMAs of 128 x 96 x 32.
__global__ void __launch_bounds__(TC5_THREADS, 1) zgemm_oz_kernel(const GemmDesc* __restrict__ descs, int prob0,
                                                                 int* status, const unsigned char* __restrict__ planes,
                                                                 int MT, int NT, int KBN, long long a_bytes,
                                                                 const int* __restrict__ ea, const int* __restrict__ fb,
                                                                 int kchunk, z* part, long long pstride, int ldp,
                                                                 int ksplit) {
    constexpr int STAGES = OZ_STAGES;
    extern __shared__ __align__(1024) unsigned char oz_smem[];
    __shared__ GemmDesc sd;
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
    const int K = part ? min(sd.k, kbeg + kchunk) : sd.k;
    const int tiles_m = (m + TC5_BM - 1) / TC5_BM;
    const int tiles_n = (n + OZ_BN - 1) / OZ_BN;
    if ((int)blockIdx.x >= tiles_m * tiles_n || K <= kbeg) {
        if (part && (int)blockIdx.x < tiles_m * tiles_n) {
            const int m0 = (blockIdx.x % tiles_m) * TC5_BM, n0 = (blockIdx.x / tiles_m) * OZ_BN;
            z* pp = part + ((long long)blockIdx.y * ksplit + blockIdx.z) * pstride;
            for (int e = threadIdx.x; e < TC5_BM * OZ_BN; e += TC5_THREADS) {
                const int i = m0 + e % TC5_BM, j = n0 + e / TC5_BM;
                if (i < m && j < n) pp[i + (long long)j * ldp] = zmk(0.0, 0.0);
            }
        }
        return;
    }
    const int tm = blockIdx.x % tiles_m, tn = blockIdx.x / tiles_m;
    const int m0 = tm * TC5_BM, n0 = tn * OZ_BN;
    const int kb0 = kbeg / OZ_KB;
    const int nkb = (K - kbeg + OZ_KB - 1) / OZ_KB;
    const long long prob = prob0 + (long long)blockIdx.y;
    const unsigned char* gA = planes + ((prob * MT + tm) * KBN + kb0) * (long long)OZ_A_BLOCK;
    const unsigned char* gB = planes + a_bytes + ((prob * NT + tn) * KBN + kb0) * (long long)OZ_B_BLOCK;

    unsigned char* stage_base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(oz_smem) + 1023) & ~uintptr_t(1023));
    const uint32_t full0 = smem_u32(&bars[0]);
    const uint32_t empty0 = smem_u32(&bars[STAGES]);
    const uint32_t done_bar = smem_u32(&bars[2 * STAGES]);

    if (tid == 0) {
        abort_flag = 0;
        for (int q = 0; q < STAGES; ++q) {
            mbar_init(full0 + 8 * q, 1);
            mbar_init(empty0 + 8 * q, 1);
        }
        mbar_init(done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"((uint32_t)OZ_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    if (warp == 0) {
        // ---------------- producer ----------------------------------------------------------------------
        bool ok = true;
        int issued = 0;
        for (int kb = 0; kb < nkb; ++kb) {
            const int q = kb % STAGES;
            if (kb >= STAGES) {
                ok = __all_sync(0xffffffffu, mbar_wait(empty0 + 8 * q, (uint32_t)(((kb / STAGES) - 1) & 1), &abort_flag));
                if (!ok) break;
            }
            if (lane == 0) {
                const uint32_t st = smem_u32(stage_base + (size_t)q * OZ_STAGE);
                mbar_arrive_expect_tx(full0 + 8 * q, (uint32_t)OZ_STAGE);
                bulk_g2s(st, gA + (long long)kb * OZ_A_BLOCK, (uint32_t)OZ_A_BLOCK, full0 + 8 * q);
                bulk_g2s(st + OZ_A_BLOCK, gB + (long long)kb * OZ_B_BLOCK, (uint32_t)OZ_B_BLOCK, full0 + 8 * q);
            }
            __syncwarp();
            issued = kb + 1;
        }
        if (!ok) {
            abort_flag = 1;
            if (lane == 0) atomicOr(status, RB_TC5_TIMEOUT);
            for (int kb = max(0, issued - STAGES); kb < issued; ++kb)
                mbar_wait(full0 + 8 * (kb % STAGES), (uint32_t)((kb / STAGES) & 1), nullptr);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------- MMA issuer --------------------------------------------------------------------
        const uint32_t idesc = oz_idesc();
        bool ok = true;
        for (int kb = 0; kb < nkb && ok; ++kb) {
            const int q = kb % STAGES;
            ok = __all_sync(0xffffffffu, mbar_wait(full0 + 8 * q, (uint32_t)((kb / STAGES) & 1), &abort_flag));
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (lane == 0) {
                const uint32_t sa = smem_u32(stage_base + (size_t)q * OZ_STAGE);
                const uint32_t sb = sa + OZ_A_BLOCK;
                constexpr uint32_t LBO_A = TC5_BM * 16, LBO_B = OZ_B_ROWS * 16, SBO = 128;
#pragma unroll
                for (int t = 2; t <= OZ_S + 1; ++t) {
                    const int jlo = t - OZ_S > 1 ? t - OZ_S : 1, jhi = t - 1 < OZ_S ? t - 1 : OZ_S;
                    const uint32_t cacc = tmem + (uint32_t)((t - 2) * OZ_MMA_N);
#pragma unroll
                    for (int j = jlo; j <= jhi; ++j) {
                        const int jp = t - j;
                        const uint32_t bp = sb + (uint32_t)((jp - 1) * OZ_B_PLANE);
                        const uint64_t Ar = umma_desc(sa + (uint32_t)((j - 1) * OZ_A_PLANE), LBO_A, SBO);
                        const uint64_t Ai = umma_desc(sa + (uint32_t)((OZ_S + j - 1) * OZ_A_PLANE), LBO_A, SBO);
                        const uint64_t Bri = umma_desc(bp + (uint32_t)(OZ_BN * 16), LBO_B, SBO);   // [Br | Bi]
                        const uint64_t Bnr = umma_desc(bp, LBO_B, SBO);                            // [-Bi | Br]
                        const uint32_t acc = (kb > 0 || j > jlo) ? 1u : 0u;
                        umma_i8(cacc, Ar, Bri, idesc, acc);
                        umma_i8(cacc, Ai, Bnr, idesc, 1u);
                    }
                }
                umma_commit(empty0 + 8 * q);
            }
            __syncwarp();
        }
        if (!ok) {
            abort_flag = 1;
            if (lane == 0) atomicOr(status, RB_TC5_TIMEOUT);
        }
        if (lane == 0) umma_commit(done_bar);
        __syncwarp();
    }

    // ---------------- epilogue: all 8 warps ----------------------------------------------------------
    const bool done = __all_sync(0xffffffffu, mbar_wait(done_bar, 0u, nullptr) && !abort_flag);
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
        const int erow = ea[(prob * MT + tm) * TC5_BM + row];
        const int* fcol = fb + (prob * NT + tn) * OZ_BN;
        const z alpha = sd.alpha, beta = sd.beta;
        z* pp = part ? part + ((long long)blockIdx.y * ksplit + blockIdx.z) * pstride : nullptr;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        constexpr double W = 1.0 / 128.0;
#pragma unroll 1
        for (int c0 = half * (OZ_BN / 2); c0 < (half + 1) * (OZ_BN / 2); c0 += 8) {
            int acc[2 * OZ_S][8];        // [t] the real parts of diagonal t + 2, [OZ_S + t] the imaginary
#pragma unroll
            for (int t = 0; t < OZ_S; ++t) {
                tmem_ld8(tmem + lane_base + (uint32_t)(t * OZ_MMA_N + c0), acc[t]);
                tmem_ld8(tmem + lane_base + (uint32_t)(t * OZ_MMA_N + OZ_BN + c0), acc[OZ_S + t]);
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (!live) continue;
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int gj = n0 + c0 + e;
                if (gj >= n) break;
                // sum_t acc_t 128^-t by Horner from the smallest weight, then the scales
                double re = (double)acc[OZ_S - 1][e], im = (double)acc[2 * OZ_S - 1][e];
#pragma unroll
                for (int t = OZ_S - 2; t >= 0; --t) {
                    re = fma(re, W, (double)acc[t][e]);
                    im = fma(im, W, (double)acc[OZ_S + t][e]);
                }
                const int p2 = erow + fcol[c0 + e] - 14;
                re = ldexp(re, p2);
                im = ldexp(im, p2);
                if (pp) {
                    pp[gi + (long long)gj * ldp] = zmk(re, im);
                    continue;
                }
                z v = zmul(alpha, zmk(re, im));
                if (use_c) zfma(v, beta, sd.C.p[cro + (long long)vcol(sd.C, gj) * sd.C.ld]);
                sd.D.p[dro + (long long)vcol(sd.D, gj) * sd.D.ld] = v;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)OZ_TMEM_COLS));
    }
}

static cudaError_t launch_oz(const GemmBatch& b, int* status, cudaStream_t s) {
    static DeviceAttrCache attr;
    cudaError_t e = ensure_smem_attr(zgemm_oz_kernel, OZ_SMEM, attr, true);
    if (e != cudaSuccess) return e;
    const OzGeom og = oz_geom(b);
    const int kchunk = (b.t5_ksplit > 1 && b.work) ? b.t5_kchunk : b.max_k;
    if (kchunk > OZ_MAX_K) return cudaErrorInvalidValue;
    unsigned char* planes = static_cast<unsigned char*>(b.t5_planes);
    int* ea = reinterpret_cast<int*>(planes + og.ea_off);
    int* fb = reinterpret_cast<int*>(planes + og.fb_off);
    // 1. row and column scales, 2. digit planes
    {
        const long long ga = (long long)b.count * (og.MT * TC5_BM / 32);
        const long long gb = ((long long)b.count * og.NT * OZ_BN + 7) / 8;
        const long long nA = (long long)b.count * og.MT * og.KBN;
        const long long nB = (long long)b.count * og.NT * og.KBN;
        if (ga > 0x7FFFFFFFLL || gb > 0x7FFFFFFFLL || nA + nB > 0x7FFFFFFFLL) return cudaErrorInvalidValue;
        e = cudaMemsetAsync(ea, 0x80, (size_t)(og.fb_off - og.ea_off), s);     // every int far below -1022
        if (e != cudaSuccess) return e;
        const unsigned gk = (unsigned)((b.max_k + OZ_SCALE_KC - 1) / OZ_SCALE_KC);
        if (gk > 65535u) return cudaErrorInvalidValue;
        oz_scale_a_kernel<<<dim3((unsigned)ga, gk), 256, 0, s>>>(b.d_desc, og.MT, ea);
        note_launch();
        oz_scale_b_kernel<<<(unsigned)gb, 256, 0, s>>>(b.d_desc, og.NT, fb);
        note_launch();
        oz_split_kernel<<<(unsigned)(nA + nB), 256, 0, s>>>(b.d_desc, og.MT, og.NT, og.KBN, nA, planes, og.a_bytes,
                                                            ea, fb);
        note_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    // 3. the products
    const int tiles = ((b.max_m + TC5_BM - 1) / TC5_BM) * ((b.max_n + OZ_BN - 1) / OZ_BN);
    if (b.t5_ksplit > 1 && b.work) {
        if (b.count > 65535 || b.t5_ksplit > 65535 || b.t5_kchunk % OZ_KB) return cudaErrorInvalidValue;
        zgemm_oz_kernel<<<dim3(tiles, b.count, b.t5_ksplit), TC5_THREADS, OZ_SMEM, s>>>(
            b.d_desc, 0, status, planes, og.MT, og.NT, og.KBN, og.a_bytes, ea, fb, b.t5_kchunk, b.work, b.t5_pstride,
            b.max_m, b.t5_ksplit);
        note_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        return launch_gemm_reduce(b, b.t5_ksplit, b.t5_pstride, s);
    }
    for (int off = 0; off < b.count; off += 65535) {
        const int cnt = (b.count - off) < 65535 ? (b.count - off) : 65535;
        zgemm_oz_kernel<<<dim3(tiles, cnt), TC5_THREADS, OZ_SMEM, s>>>(b.d_desc + off, off, status, planes, og.MT,
                                                                       og.NT, og.KBN, og.a_bytes, ea, fb, 0, nullptr,
                                                                       0, 0, 1);
        note_launch();
    }
    return cudaGetLastError();
}

// ================= host: engine choice, split-K plans, workspaces, dispatch =========================

int tc5_engine(const GemmBatch& b) {
    if (b.t5_engine == TC5_ENGINE_TF32X3 || b.t5_engine == TC5_ENGINE_INT8) return b.t5_engine;
    static const int dflt = [] {
        const char* v = std::getenv("RB_MIXED_ENGINE");
        return (v && std::strcmp(v, "tf32x3") == 0) ? TC5_ENGINE_TF32X3 : TC5_ENGINE_INT8;
    }();
    return dflt;
}

// k granularity and output columns per tile of a batch's engine
static int t5_kblock(const GemmBatch& b) { return tc5_engine(b) == TC5_ENGINE_INT8 ? OZ_KB : TC5_KB; }

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
    const int kq = t5_kblock(b);
    const int kc = (int)(((b.max_k + sp - 1) / sp + kq - 1) / kq * kq);
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
    const int kq = t5_kblock(b);
    const int kc = (int)(((b.max_k + sp - 1) / sp + kq - 1) / kq * kq);
    const int ks = (b.max_k + kc - 1) / kc;
    if (ks < 2) return 0;
    b.t5_kchunk = kc;
    b.t5_ksplit = ks;
    b.t5_pstride = (long long)b.max_m * b.max_n;
    return (long long)b.count * ks * b.t5_pstride;
}

int tc5_tile_n(const GemmBatch& b) {
    if (tc5_engine(b) == TC5_ENGINE_INT8) return OZ_BN;
    // RB_TC5_BN (32, 64, 128 or 256; read at every call) overrides the rule, for measurements
    if (const char* v = std::getenv("RB_TC5_BN")) {
        const int f = std::atoi(v);
        if (f == 32 || f == 64 || f == 128 || f == 256) return f;
    }
    // n columns per tile: 32 / 64 for the narrow solve products; 256 where the 128 x 256 tiles
    // still fill a wave of the 148 SMs (each A block then serves twice the columns), else 128
    if (b.max_n <= 32) return 32;
    if (b.max_n <= 64) return 64;
    const long long tm = (long long)b.count * ((b.max_m + TC5_BM - 1) / TC5_BM);
    if (tm * ((b.max_n + 255) / 256) >= 148) return 256;
    return 128;
}

size_t tc5_plane_bytes(const GemmBatch& b) {
    if (b.count == 0 || b.max_m == 0 || b.max_n == 0 || b.max_k == 0) return 0;
    if (tc5_engine(b) == TC5_ENGINE_INT8) return (size_t)oz_geom(b).total;
    const int bn = tc5_tile_n(b);
    const PlaneGeom pg = plane_geom(b, bn);
    return (size_t)pg.a_bytes + (size_t)b.count * pg.NT * pg.KBN * (size_t)bn * TC5_KB * 16;
}

cudaError_t launch_gemm_tc5(const GemmBatch& b, int* status, cudaStream_t s) {
    if (b.count == 0 || b.max_m == 0 || b.max_n == 0) return cudaSuccess;
    if (!status || !b.t5_planes || (reinterpret_cast<uintptr_t>(b.t5_planes) & 255) ||
        tc5_plane_bytes(b) > b.t5_plane_cap)
        return cudaErrorInvalidValue;
    if (tc5_engine(b) == TC5_ENGINE_INT8) return launch_oz(b, status, s);
    const int bn = tc5_tile_n(b);
    if (bn == 32) return launch_tc5<32>(b, status, s);
    if (bn == 64) return launch_tc5<64>(b, status, s);
    if (bn == 256) return launch_tc5<256>(b, status, s);
    return launch_tc5<128>(b, status, s);
}

}  // namespace rb
