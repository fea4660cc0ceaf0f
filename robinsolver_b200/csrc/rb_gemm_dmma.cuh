// rb_gemm_dmma.cuh -- one C tile of a complex128 GEMM on the FP64 tensor-core instruction
// (mma.sync.aligned.m8n8k4.f64), for the large merge GEMMs.
//
// A complex product takes three real MMAs (the 3M method): P1 += Ar Br, P2 += Ai Bi,
// P3 += (Ar + Ai)(Br + Bi), and the epilogue forms Re = P1 - P2, Im = P3 - P1 - P2.  Against the
// four-product form this saves a quarter of the tensor-core work for an error bound about twice
// as large, still normwise: |error| <= c k u |A| |B| entrywise in the moduli.  The CTA tile is
// BM x BN complex with 8 warps in a WM x WN grid; each warp owns a (BM/WM) x (BN/WN) tile of 8x8
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
        for (int k4 = 0; k4 < BK; k4 += 4) {
            double far[TMW], fai[TMW], fas[TMW], fbr[TNW], fbi[TNW], fbs[TNW];
#pragma unroll
            for (int i = 0; i < TMW; ++i) {
                const z a = As[(k4 + lc) * LDA + wrow0 + i * 8 + lr];
                far[i] = a.x;
                fai[i] = a.y;
                fas[i] = a.x + a.y;
            }
#pragma unroll
            for (int j = 0; j < TNW; ++j) {
                const z b = Bs[(k4 + lc) * LDB + wcol0 + j * 8 + lr];
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
    }
    cp_async_wait<0>();

    const z alpha = sd.alpha, beta = sd.beta;
    const ZView C = sd.C;
    const ZOut D = sd.D;
#pragma unroll
    for (int i = 0; i < TMW; ++i) {
        const int gi = m0 + wrow0 + i * 8 + lr;
        if (gi >= m) continue;
        const long long drow = (long long)vrow(D, gi);
        const bool use_c = C.p && !(gi >= sd.nobeta_r0 && gi < sd.nobeta_r1);
        const long long crow = use_c ? (long long)vrow(C, gi) : 0;
#pragma unroll
        for (int j = 0; j < TNW; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gj = n0 + wcol0 + j * 8 + 2 * lc + h;
                if (gj >= n) continue;
                const double re = p1[i][j][h] - p2[i][j][h];
                const double im = p3[i][j][h] - p1[i][j][h] - p2[i][j][h];
                z v = zmul(alpha, zmk(re, im));
                if (use_c) {
                    const z c = C.p[crow + (long long)vcol(C, gj) * C.ld];
                    zfma(v, beta, c);
                }
                D.p[drow + (long long)vcol(D, gj) * D.ld] = v;
            }
    }
}

}  // namespace rb
