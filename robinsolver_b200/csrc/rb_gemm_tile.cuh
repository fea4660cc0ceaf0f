// rb_gemm_tile.cuh -- one C tile of a complex128 GEMM problem described by a GemmDesc that
// already sits in shared memory.  Used by the descriptor-batched GEMM (rb_gemm.cu) and by the
// blocked Gauss-Jordan update (rb_gj.cu), which builds its descriptor inside the kernel.
//
// Thread (tr, tc) owns rows tr + i*RG and columns tc + j*CG of the BM x BN tile (strided so
// that a warp's epilogue stores and shared-memory operand reads are contiguous).  Operand
// tiles go global -> registers -> shared memory with one tile of look-ahead; the inner loop is
// 4 DFMA per complex multiply-add.
#pragma once
#include "rb_common.cuh"

namespace rb {

template <int BM, int BN, int TM, int TN, int BK>
__device__ __forceinline__ void zgemm_tile(const GemmDesc& sd, int tile) {
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int RG = BM / TM;
    constexpr int CG = BN / TN;
    constexpr int A_PER = BM * BK / NT;
    constexpr int B_PER = BK * BN / NT;
    static_assert(NT % BM == 0 && NT % BK == 0, "tile/thread mismatch");
    static_assert(A_PER * NT == BM * BK && B_PER * NT == BK * BN, "tile/thread mismatch");

    __shared__ z As[2][BK][BM];
    __shared__ z Bs[2][BK][BN];

    const int tid = threadIdx.x;
    const int m = sd.m, n = sd.n, K = sd.k;
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

    z ra[A_PER], rbv[B_PER];
    auto gload = [&](int k0) {
#pragma unroll
        for (int e = 0; e < A_PER; ++e) {
            const int gk = k0 + akk0 + e * (NT / BM);
            ra[e] = (arow_ok && gk < K) ? A.p[arow + (long long)vcol(A, gk) * A.ld] : zmk(0.0, 0.0);
        }
        const int gk = k0 + bkk;
        const bool kok = gk < K;
        const long long brow = kok ? (long long)vrow(B, gk) : 0;
#pragma unroll
        for (int e = 0; e < B_PER; ++e)
            rbv[e] = (kok && bcol_ok[e]) ? B.p[brow + bcol[e]] : zmk(0.0, 0.0);
    };
    auto sstore = [&](int buf) {
#pragma unroll
        for (int e = 0; e < A_PER; ++e) As[buf][akk0 + e * (NT / BM)][ai] = ra[e];
#pragma unroll
        for (int e = 0; e < B_PER; ++e) Bs[buf][bkk][bj0 + e * (NT / BK)] = rbv[e];
    };

    const int tr = tid % RG;
    const int tc = tid / RG;
    z acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = zmk(0.0, 0.0);

    gload(0);
    sstore(0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += BK) {
        const bool more = (k0 + BK) < K;
        if (more) gload(k0 + BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            z a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[buf][kk][tr + i * RG];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = Bs[buf][kk][tc + j * CG];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) zfma(acc[i][j], a[i], b[j]);
        }
        if (more) sstore(buf ^ 1);
        __syncthreads();
        buf ^= 1;
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

// thread-block sizes of the tile configurations
template <int BM, int BN, int TM, int TN>
struct TileThreads { static constexpr int value = (BM / TM) * (BN / TN); };

}  // namespace rb
