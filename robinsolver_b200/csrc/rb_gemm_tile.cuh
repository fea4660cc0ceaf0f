// rb_gemm_tile.cuh -- one C tile of a complex128 GEMM problem on DFMA register tiles, for the small
// merge GEMMs and every solve GEMM (rb_gemm.cu).
//
// Thread (tr, tc) owns rows tr + i*RG and columns tc + j*CG of the BM x BN tile (strided so
// that a warp's epilogue stores and shared-memory operand reads are contiguous).  Operand tiles
// stream global -> shared memory with cp.async in a STAGES-deep ring, so that STAGES-1 k-tiles
// are in flight while one is multiplied (the skinny solve GEMMs, k ~ 1000 and n ~ 32, are
// load-latency bound otherwise).  The inner loop is 4 DFMA per complex multiply-add, and every
// element sums its products in k order: results do not depend on the tile shape.
#pragma once
#include "rb_common.cuh"
#include "rb_gemm_dmma.cuh"    // cp.async helpers

namespace rb {

template <int BM, int BN, int BK, int STAGES>
struct DfmaCfg {
    static constexpr int STAGE_Z = BK * BM + BK * BN;
    static constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE_Z * sizeof(z);
};

// With PARTIAL, only k in [kbeg, kend) is summed and the raw sums go to part (element (i, j) at
// part[i + j * ldp]) for a later fixed-order reduction over the k ranges (split-K).
template <int BM, int BN, int TM, int TN, int BK, int STAGES, bool PARTIAL = false>
__device__ __forceinline__ void zgemm_tile(const GemmDesc& sd, int tile, z* smem, int kbeg = 0, int kend = 0,
                                           z* part = nullptr, int ldp = 0) {
    using Cfg = DfmaCfg<BM, BN, BK, STAGES>;
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int RG = BM / TM;
    constexpr int CG = BN / TN;
    constexpr int A_PER = BM * BK / NT;
    constexpr int B_PER = BK * BN / NT;
    static_assert(NT % BM == 0 && NT % BK == 0, "tile/thread mismatch");
    static_assert(A_PER * NT == BM * BK && B_PER * NT == BK * BN, "tile/thread mismatch");

    const int tid = threadIdx.x;
    const int m = sd.m, n = sd.n;
    const int K = PARTIAL ? min(sd.k, kend) : sd.k;
    const int kb0 = PARTIAL ? kbeg : 0;
    const int tiles_m = (m + BM - 1) / BM;
    const int tmi = tile % tiles_m;
    const int tni = tile / tiles_m;
    if (tni * BN >= n || m <= 0) return;      // uniform across the CTA
    const int m0 = tmi * BM, n0 = tni * BN;

    const ZView A = sd.A;
    const ZView B = sd.B;

    const int ai = tid % BM;
    const int akk0 = tid / BM;
    const int bkk = tid % BK;
    const int bj0 = tid / BK;
    const bool arow_ok = (m0 + ai) < m;
    const long long arow = arow_ok ? (long long)vrow(A, m0 + ai) : 0;
    long long bcol[B_PER];
    bool bcol_ok[B_PER];
#pragma unroll
    for (int e = 0; e < B_PER; ++e) {
        const int j = n0 + bj0 + e * (NT / BK);
        bcol_ok[e] = j < n;
        bcol[e] = bcol_ok[e] ? (long long)vcol(B, j) * B.ld : 0;
    }
    const int ktiles = K > kb0 ? (K - kb0 + BK - 1) / BK : 0;
    auto issue = [&](int kt) {
        z* As = smem + (kt % STAGES) * Cfg::STAGE_Z;
        z* Bs = As + BK * BM;
        const int k0 = kb0 + kt * BK;
#pragma unroll
        for (int e = 0; e < A_PER; ++e) {
            const int kk = akk0 + e * (NT / BM);
            const int gk = k0 + kk;
            const bool ok = arow_ok && gk < K;
            const z* src = ok ? A.p + arow + (long long)vcol(A, gk) * A.ld : A.p;
            cp_async16(As + kk * BM + ai, src, ok ? 16 : 0);
        }
        const int gk = k0 + bkk;
        const bool kok = gk < K;
        const long long brow = kok ? (long long)vrow(B, gk) : 0;
#pragma unroll
        for (int e = 0; e < B_PER; ++e) {
            const bool ok = kok && bcol_ok[e];
            const z* src = ok ? B.p + brow + bcol[e] : B.p;
            cp_async16(Bs + bkk * BN + bj0 + e * (NT / BK), src, ok ? 16 : 0);
        }
    };

    const int tr = tid % RG;
    const int tc = tid / RG;
    z acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = zmk(0.0, 0.0);

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < ktiles) issue(s);
        cp_async_commit();
    }
    for (int kt = 0; kt < ktiles; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();                 // tile kt visible; everyone is done with tile kt-1's stage
        if (kt + STAGES - 1 < ktiles) issue(kt + STAGES - 1);
        cp_async_commit();
        const z* As = smem + (kt % STAGES) * Cfg::STAGE_Z;
        const z* Bs = As + BK * BM;
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            z a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[kk * BM + tr + i * RG];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = Bs[kk * BN + tc + j * CG];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) zfma(acc[i][j], a[i], b[j]);
        }
    }
    cp_async_wait<0>();

    if (PARTIAL) {
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            const int gi = m0 + tr + i * RG;
            if (gi >= m) continue;
#pragma unroll
            for (int j = 0; j < TN; ++j) {
                const int gj = n0 + tc + j * CG;
                if (gj < n) part[gi + (long long)gj * ldp] = acc[i][j];
            }
        }
        return;
    }
    const z alpha = sd.alpha, beta = sd.beta;
    const ZView C = sd.C;
    const ZOut D = sd.D;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int gi = m0 + tr + i * RG;
        if (gi >= m) continue;
        const long long drow = (long long)vrow(D, gi);
        const bool use_c = C.p && !(gi >= sd.nobeta_r0 && gi < sd.nobeta_r1);
        const long long crow = use_c ? (long long)vrow(C, gi) : 0;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int gj = n0 + tc + j * CG;
            if (gj >= n) continue;
            z v = zmul(alpha, acc[i][j]);
            if (use_c) {
                const z c = C.p[crow + (long long)vcol(C, gj) * C.ld];
                zfma(v, beta, c);
            }
            D.p[drow + (long long)vcol(D, gj) * D.ld] = v;
        }
    }
}

}  // namespace rb
