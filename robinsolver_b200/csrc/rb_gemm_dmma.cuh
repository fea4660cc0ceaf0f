// rb_gemm_dmma.cuh -- one C tile of a complex128 GEMM on the FP64 tensor-core instruction
// (mma.sync.aligned.m8n8k4.f64), for the large merge GEMMs.
//
// A complex product takes three real MMAs (the 3M method): P1 += Ar Br, P2 += Ai Bi,
// P3 += (Ar + Ai)(Br + Bi), and the epilogue forms Re = P1 - P2, Im = P3 - P1 - P2.  Against the
// four-product form this saves a quarter of the tensor-core work for an error bound about twice
// as large, still normwise: |error| <= c k u |A| |B| entrywise in the moduli.  The CTA tile is
// BM x BN complex with WM x WN warps; each warp owns a (BM/WM) x (BN/WN) tile of 8x8
// MMA tiles, accumulated in registers.  Operand tiles stream global -> shared memory with
// cp.async in a STAGES-deep ring (the loads of STAGES-1 future k-tiles are in flight while one is
// multiplied), complex elements kept interleaved so that one 16-byte shared load yields both
// planes of a fragment element.  Rows of a stage are padded by 2 complex elements, which puts the
// 8 lanes of each quarter-warp's fragment loads in 8 distinct 16-byte bank groups.
//
// Fragment layout of m8n8k4 with .f64 (PTX ISA): A (8x4, row) -- lane holds (lane>>2, lane&3);
// B (4x8, col) -- lane holds (lane&3, lane>>2); C/D (8x8) -- lane holds (lane>>2, 2*(lane&3)+{0,1}).
#pragma once
#include "rb_common.cuh"

namespace rb {

// not volatile: the compiler may interleave independent MMAs to hide the MMA latency
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

// 16-byte asynchronous global -> shared copy; src_bytes = 0 fills the destination with zeros
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// D = alpha (P1 - P2 + i (P3 - P1 - P2)) + beta C for one warp's TMW x TNW MMA tiles, whose
// top-left element is (r0, c0).  Column offsets are looked up once, and each row's C elements are
// all loaded before any of its D elements is stored, so that the loads overlap: C aliases D, if
// at all, element for element, so no store can change a C element that is read later.
template <int TMW, int TNW>
__device__ __forceinline__ void dmma_store(const GemmDesc& sd, const double (&p1)[TMW][TNW][2],
                                           const double (&p2)[TMW][TNW][2], const double (&p3)[TMW][TNW][2],
                                           int r0, int c0, int lr, int lc) {
    const int m = sd.m, n = sd.n;
    const z alpha = sd.alpha, beta = sd.beta;
    const ZView C = sd.C;
    const ZOut D = sd.D;
    int dcol[TNW][2], ccol[TNW][2];      // output / C column indices; -1: beyond n
#pragma unroll
    for (int j = 0; j < TNW; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int gj = c0 + j * 8 + 2 * lc + h;
            const bool ok = gj < n;
            dcol[j][h] = ok ? vcol(D, gj) : -1;
            ccol[j][h] = ok && C.p ? vcol(C, gj) : 0;
        }
#pragma unroll
    for (int i = 0; i < TMW; ++i) {
        const int gi = r0 + i * 8 + lr;
        if (gi >= m) continue;
        const long long drow = (long long)vrow(D, gi);
        const bool use_c = C.p && !(gi >= sd.nobeta_r0 && gi < sd.nobeta_r1);
        const long long crow = use_c ? (long long)vrow(C, gi) : 0;
        z c[TNW][2];
#pragma unroll
        for (int j = 0; j < TNW; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h)
                c[j][h] = (use_c && dcol[j][h] >= 0) ? C.p[crow + (long long)ccol[j][h] * C.ld] : zmk(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < TNW; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (dcol[j][h] < 0) continue;
                const double re = p1[i][j][h] - p2[i][j][h];
                const double im = p3[i][j][h] - p1[i][j][h] - p2[i][j][h];
                z v = zmul(alpha, zmk(re, im));
                if (use_c) zfma(v, beta, c[j][h]);
                D.p[drow + (long long)dcol[j][h] * D.ld] = v;
            }
    }
}

// one k-step of 4 of the 3M product on a warp's TMW x TNW MMA tiles; As and Bs point at this
// lane's first fragment element in the A and B stages (MMA tiles 8 elements apart)
template <int TMW, int TNW, int LDA, int LDB>
__device__ __forceinline__ void dmma_k4(const z* __restrict__ As, const z* __restrict__ Bs, double (&p1)[TMW][TNW][2],
                                        double (&p2)[TMW][TNW][2], double (&p3)[TMW][TNW][2]) {
    double far[TMW], fai[TMW], fas[TMW], fbr[TNW], fbi[TNW], fbs[TNW];
#pragma unroll
    for (int i = 0; i < TMW; ++i) {
        const z a = As[i * 8];
        far[i] = a.x;
        fai[i] = a.y;
        fas[i] = a.x + a.y;
    }
#pragma unroll
    for (int j = 0; j < TNW; ++j) {
        const z b = Bs[j * 8];
        fbr[j] = b.x;
        fbi[j] = b.y;
        fbs[j] = b.x + b.y;
    }
    // three passes over the warp tile so that two MMAs on one accumulator are never adjacent
#pragma unroll
    for (int i = 0; i < TMW; ++i)
#pragma unroll
        for (int j = 0; j < TNW; ++j) dmma884(p1[i][j][0], p1[i][j][1], far[i], fbr[j]);
#pragma unroll
    for (int i = 0; i < TMW; ++i)
#pragma unroll
        for (int j = 0; j < TNW; ++j) dmma884(p2[i][j][0], p2[i][j][1], fai[i], fbi[j]);
#pragma unroll
    for (int i = 0; i < TMW; ++i)
#pragma unroll
        for (int j = 0; j < TNW; ++j) dmma884(p3[i][j][0], p3[i][j][1], fas[i], fbs[j]);
}

template <int BM, int BN, int WM, int WN>
struct DmmaCfg {
    static constexpr int NT = 32 * WM * WN;     // threads
    static constexpr int BK = 8;                // complex k per stage (2 MMA k-steps)
    static constexpr int STAGES = 4;
    static constexpr int LDA = BM + 2;          // complex elements per k-row of an A stage
    static constexpr int LDB = BN + 2;
    static constexpr int TMW = BM / WM / 8;     // MMA tiles per warp along M
    static constexpr int TNW = BN / WN / 8;     // ... along N
    static constexpr int STAGE_Z = BK * LDA + BK * LDB;
    static constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE_Z * sizeof(z);
};

template <int BM, int BN, int WM, int WN>
__device__ __forceinline__ void zgemm_tile_dmma(const GemmDesc& sd, int tile, z* smem) {
    using Cfg = DmmaCfg<BM, BN, WM, WN>;
    constexpr int NT = Cfg::NT, BK = Cfg::BK, LDA = Cfg::LDA, LDB = Cfg::LDB, STAGES = Cfg::STAGES;
    constexpr int TMW = Cfg::TMW, TNW = Cfg::TNW;
    constexpr int A_PER = BM * BK / NT;
    constexpr int B_PER = BK * BN / NT;
    static_assert(A_PER * NT == BM * BK && B_PER * NT == BK * BN, "tile/thread mismatch");
    static_assert(NT % BM == 0 && NT % BK == 0, "tile/thread mismatch");

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int m = sd.m, n = sd.n, K = sd.k;
    const int tiles_m = (m + BM - 1) / BM;
    const int tmi = tile % tiles_m;
    const int tni = tile / tiles_m;
    if (tni * BN >= n || m <= 0) return;
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
    const int ktiles = (K + BK - 1) / BK;
    auto issue = [&](int kt) {
        z* As = smem + (kt % STAGES) * Cfg::STAGE_Z;
        z* Bs = As + BK * LDA;
        const int k0 = kt * BK;
#pragma unroll
        for (int e = 0; e < A_PER; ++e) {
            const int kk = akk0 + e * (NT / BM);
            const int gk = k0 + kk;
            const bool ok = arow_ok && gk < K;
            const z* src = ok ? A.p + arow + (long long)vcol(A, gk) * A.ld : A.p;
            cp_async16(As + kk * LDA + ai, src, ok ? 16 : 0);
        }
        const int gk = k0 + bkk;
        const bool kok = gk < K;
        const long long brow = kok ? (long long)vrow(B, gk) : 0;
#pragma unroll
        for (int e = 0; e < B_PER; ++e) {
            const bool ok = kok && bcol_ok[e];
            const z* src = ok ? B.p + brow + bcol[e] : B.p;
            cp_async16(Bs + bkk * LDB + bj0 + e * (NT / BK), src, ok ? 16 : 0);
        }
    };

    const int wm = warp % WM, wn = warp / WM;
    const int wrow0 = wm * (BM / WM), wcol0 = wn * (BN / WN);
    const int lr = lane >> 2, lc = lane & 3;
    double p1[TMW][TNW][2], p2[TMW][TNW][2], p3[TMW][TNW][2];
#pragma unroll
    for (int i = 0; i < TMW; ++i)
#pragma unroll
        for (int j = 0; j < TNW; ++j) {
            p1[i][j][0] = p1[i][j][1] = 0.0;
            p2[i][j][0] = p2[i][j][1] = 0.0;
            p3[i][j][0] = p3[i][j][1] = 0.0;
        }

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
        const z* Bs = As + BK * LDA;
#pragma unroll
        for (int k4 = 0; k4 < BK; k4 += 4)
            dmma_k4<TMW, TNW, LDA, LDB>(As + (k4 + lc) * LDA + wrow0 + lr, Bs + (k4 + lc) * LDB + wcol0 + lr, p1, p2, p3);
    }
    cp_async_wait<0>();
    dmma_store<TMW, TNW>(sd, p1, p2, p3, m0 + wrow0, n0 + wcol0, lr, lc);
}

// The same product for batches whose k runs contiguously through both operands
// (gemm_k_contiguous): each thread's copy sources advance by a fixed stride per k-tile, the stage
// ring is walked with running indices, and only the last partial k-tile is predicated.  This
// halves the instructions issued per MMA against the general tile, whose per-element map and
// band look-ups dominate its issue slots; with 32x32 warp tiles (4 warps, 96 accumulators a
// thread, two CTAs per SM) the MMA pipe stays busy 87% of the time on the large merges, where
// the general tile reaches 74%.
template <int BM, int BN, int WM, int WN, int BK, int STAGES>
struct DmmaKcCfg {
    static constexpr int NT = 32 * WM * WN;
    static constexpr int LDA = BM + 2, LDB = BN + 2;
    static constexpr int TMW = BM / WM / 8, TNW = BN / WN / 8;
    static constexpr int STAGE_Z = BK * LDA + BK * LDB;
    static constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE_Z * sizeof(z);
};

template <int BM, int BN, int WM, int WN, int BK, int STAGES>
__device__ __forceinline__ void zgemm_tile_dmma_kc(const GemmDesc& sd, int tile, z* smem) {
    using Cfg = DmmaKcCfg<BM, BN, WM, WN, BK, STAGES>;
    constexpr int NT = Cfg::NT, LDA = Cfg::LDA, LDB = Cfg::LDB, TMW = Cfg::TMW, TNW = Cfg::TNW;
    constexpr int STAGE_Z = Cfg::STAGE_Z;
    constexpr int A_PER = BM * BK / NT, B_PER = BK * BN / NT;
    static_assert(A_PER * NT == BM * BK && B_PER * NT == BK * BN, "tile/thread mismatch");
    static_assert(NT % BM == 0 && NT % BK == 0 && BK % 4 == 0, "tile/thread mismatch");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m = sd.m, n = sd.n, K = sd.k;
    const int tiles_m = (m + BM - 1) / BM;
    const int tmi = tile % tiles_m, tni = tile / tiles_m;
    if (tni * BN >= n || m <= 0) return;
    const int m0 = tmi * BM, n0 = tni * BN;
    const ZView A = sd.A, B = sd.B;

    // this thread copies A rows ai, k-rows akk0 + e NT/BM, and B k-row bkk, columns bj0 + e NT/BK
    const int ai = tid % BM, akk0 = tid / BM, bkk = tid % BK, bj0 = tid / BK;
    const bool arow_ok = (m0 + ai) < m;
    const z* a_src = A.p + (arow_ok ? (long long)vrow(A, m0 + ai) : 0) + (long long)akk0 * A.ld;
    const long long a_es = (long long)(NT / BM) * A.ld, a_ks = (long long)BK * A.ld;
    const int a_bytes = arow_ok ? 16 : 0;
    const z* b_src[B_PER];
    bool bcol_ok[B_PER];
#pragma unroll
    for (int e = 0; e < B_PER; ++e) {
        const int j = n0 + bj0 + e * (NT / BK);
        bcol_ok[e] = j < n;
        b_src[e] = B.p + (bcol_ok[e] ? (long long)vcol(B, j) * B.ld : 0) + bkk;
    }
    const int ktiles = (K + BK - 1) / BK, kfull = K / BK;
    const int a_dst = akk0 * LDA + ai;
    const int b_dst = BK * LDA + bkk * LDB + bj0;
    auto issue = [&](int kt, int stage) {
        z* S = smem + stage * STAGE_Z;
        const long long ka = (long long)kt * a_ks;
        const int kb = kt * BK;
        if (kt < kfull) {
#pragma unroll
            for (int e = 0; e < A_PER; ++e) cp_async16(S + a_dst + e * (NT / BM) * LDA, a_src + ka + e * a_es, a_bytes);
#pragma unroll
            for (int e = 0; e < B_PER; ++e) cp_async16(S + b_dst + e * (NT / BK), b_src[e] + kb, bcol_ok[e] ? 16 : 0);
        } else {
#pragma unroll
            for (int e = 0; e < A_PER; ++e) {
                const bool ok = arow_ok && kb + akk0 + e * (NT / BM) < K;
                cp_async16(S + a_dst + e * (NT / BM) * LDA, ok ? a_src + ka + e * a_es : A.p, ok ? 16 : 0);
            }
            const bool kok = kb + bkk < K;
#pragma unroll
            for (int e = 0; e < B_PER; ++e) {
                const bool ok = kok && bcol_ok[e];
                cp_async16(S + b_dst + e * (NT / BK), ok ? b_src[e] + kb : B.p, ok ? 16 : 0);
            }
        }
    };

    const int wm = warp % WM, wn = warp / WM;
    const int wrow0 = wm * (BM / WM), wcol0 = wn * (BN / WN);
    const int lr = lane >> 2, lc = lane & 3;
    const int fa = lc * LDA + wrow0 + lr;
    const int fb = BK * LDA + lc * LDB + wcol0 + lr;
    double p1[TMW][TNW][2], p2[TMW][TNW][2], p3[TMW][TNW][2];
#pragma unroll
    for (int i = 0; i < TMW; ++i)
#pragma unroll
        for (int j = 0; j < TNW; ++j) {
            p1[i][j][0] = p1[i][j][1] = 0.0;
            p2[i][j][0] = p2[i][j][1] = 0.0;
            p3[i][j][0] = p3[i][j][1] = 0.0;
        }
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < ktiles) issue(s, s);
        cp_async_commit();
    }
    int rs = 0, ws = STAGES - 1;
    for (int kt = 0; kt < ktiles; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();                 // tile kt visible; everyone is done with tile kt-1's stage
        if (kt + STAGES - 1 < ktiles) issue(kt + STAGES - 1, ws);
        cp_async_commit();
        ws = ws + 1 == STAGES ? 0 : ws + 1;
        const z* S = smem + rs * STAGE_Z;
        rs = rs + 1 == STAGES ? 0 : rs + 1;
#pragma unroll
        for (int k4 = 0; k4 < BK; k4 += 4) dmma_k4<TMW, TNW, LDA, LDB>(S + fa + k4 * LDA, S + fb + k4 * LDB, p1, p2, p3);
    }
    cp_async_wait<0>();
    dmma_store<TMW, TNW>(sd, p1, p2, p3, m0 + wrow0, n0 + wcol0, lr, lc);
}

}  // namespace rb
