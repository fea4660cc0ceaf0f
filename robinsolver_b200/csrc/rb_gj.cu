// rb_gj.cu -- batched in-place Gauss-Jordan inversion of complex128 matrices for sm_100a.
//
// The reference forms inv(D) explicitly (zgetri after zgetrf, robin_tree_module.f90:449-455)
// and applies D and S through their LU factors.  Here every dense inverse the factor/solve
// needs (the leaf's interior Schur complement, D and S of each merge) is formed explicitly by
// Gauss-Jordan elimination with partial pivoting, so that later applications are GEMMs.
// Pivots are chosen as LAPACK's izamax does: largest |re|+|im| in the column, first on ties.
//
// m <= 64: one CTA per matrix holds the whole matrix in shared memory.
// m  > 64: blocked Gauss-Jordan.  Per panel of nb columns:
//   1. gj_panel: one CTA per matrix, one matrix row per thread in registers, runs the
//      unblocked elimination on the panel (pivot search below the diagonal, row exchange,
//      scaling, elimination of every other row), leaving the accumulated transform W in the
//      panel columns;
//   2. gj_swapcopy: applies the panel's row exchanges to every other column and copies the
//      panel rows Z = A[P, rest];
//   3. gj_update: A[i, rest] += W[i,:] Z for rows outside the panel and A[P, rest] = W_P Z for
//      the panel rows, one GEMM on the shared tile engine.  (Writing the panel rows as
//      Z + (W_P - I) Z instead cancels catastrophically: W_P's diagonal holds the reciprocal
//      pivots, ~h^2 for the FD matrices here.)
// After the last panel the column exchanges are undone in reverse order (gj_unscramble).
#include "rb_gemm_tile.cuh"
#include "rb_kernels.h"

namespace rb {

int gj_panel_width(int m) {
    if (m <= GJ_SMALL_MAX) return 0;
    if (m <= 256) return 16;
    return 8;
}

long long gj_workspace_elems(int m) {
    const int nb = gj_panel_width(m);
    return nb == 0 ? 0 : (long long)m * nb;
}

// warp argmax: larger value wins, equal values go to the smaller index
__device__ __forceinline__ void argmax_warp(double& v, int& i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, v, o);
        const int oi = __shfl_down_sync(0xffffffffu, i, o);
        if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
    }
}

__device__ __forceinline__ bool zis0(z a) { return a.x == 0.0 && a.y == 0.0; }

// ---------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) gj_small_kernel(const GJDesc* __restrict__ descs, int m,
                                                       int* status) {
    extern __shared__ z S[];                  // m*m, column-major
    __shared__ z fcol[GJ_SMALL_MAX];
    __shared__ int ipiv[GJ_SMALL_MAX];
    __shared__ int sp;
    const GJDesc g = descs[blockIdx.x];
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < m * m; e += nt) {
        const int r = e % m, c = e / m;
        S[e] = g.A[r + (long long)c * g.ld];
    }
    __syncthreads();
    bool bad = false;
    for (int k = 0; k < m; ++k) {
        if (tid < 32) {
            double best = -1.0;
            int bi = m;
            for (int r = k + tid; r < m; r += 32) {
                const double v = zabs1(S[r + k * m]);
                if (v > best) { best = v; bi = r; }
            }
            argmax_warp(best, bi);
            if (tid == 0) { sp = bi; ipiv[k] = bi; }
        }
        __syncthreads();
        const int p = sp;
        if (p != k)
            for (int c = tid; c < m; c += nt) {
                const z t = S[k + c * m];
                S[k + c * m] = S[p + c * m];
                S[p + c * m] = t;
            }
        __syncthreads();
        const z piv = S[k + k * m];
        const z pinv = zrcp(piv);
        if (zis0(piv)) bad = true;
        for (int i = tid; i < m; i += nt) fcol[i] = S[i + k * m];
        __syncthreads();
        for (int c = tid; c < m; c += nt) S[k + c * m] = (c == k) ? pinv : zmul(S[k + c * m], pinv);
        __syncthreads();
        for (int e = tid; e < m * m; e += nt) {
            const int i = e % m, c = e / m;
            if (i == k) continue;
            const z f = fcol[i];
            if (c == k) S[e] = zneg(zmul(f, pinv));
            else zfms(S[e], f, S[k + c * m]);
        }
        __syncthreads();
    }
    // undo the column exchanges, last first; each thread owns whole rows
    for (int r = tid; r < m; r += nt)
        for (int k = m - 1; k >= 0; --k) {
            const int p = ipiv[k];
            if (p != k) {
                const z t = S[r + k * m];
                S[r + k * m] = S[r + p * m];
                S[r + p * m] = t;
            }
        }
    __syncthreads();
    for (int e = tid; e < m * m; e += nt) {
        const int r = e % m, c = e / m;
        g.A[r + (long long)c * g.ld] = S[e];
    }
    if (bad && tid == 0) atomicOr(status, 1);
}

// ---------------------------------------------------------------------------------------------------
// MAXT: largest matrix (= threads per CTA) a panel instance serves; it bounds the registers
// available to row[NB]
template <int NB, int MAXT>
__global__ void __launch_bounds__(MAXT) gj_panel_kernel(const GJDesc* __restrict__ descs, int m,
                                                        int k0, int nbk, int* status) {
    __shared__ z xa[NB], xb[NB], prow[NB];
    __shared__ double wv[32];
    __shared__ int wi[32];
    __shared__ int s_p;
    const GJDesc g = descs[blockIdx.x];
    const int r = threadIdx.x;
    const bool own = r < m;
    const int lane = r & 31, warp = r >> 5, nwarps = (blockDim.x + 31) >> 5;
    z row[NB];
#pragma unroll
    for (int kk = 0; kk < NB; ++kk)
        row[kk] = (own && kk < nbk) ? g.A[r + (long long)(k0 + kk) * g.ld] : zmk(0.0, 0.0);
    bool bad = false;
#pragma unroll
    for (int kk = 0; kk < NB; ++kk) {
        if (kk >= nbk) break;
        const int c = k0 + kk;
        double v = (own && r >= c) ? zabs1(row[kk]) : -1.0;
        int idx = own ? r : 0x7fffffff;
        argmax_warp(v, idx);
        if (lane == 0) { wv[warp] = v; wi[warp] = idx; }
        __syncthreads();
        if (warp == 0) {
            v = lane < nwarps ? wv[lane] : -1.0;
            idx = lane < nwarps ? wi[lane] : 0x7fffffff;
            argmax_warp(v, idx);
            if (lane == 0) s_p = idx;
        }
        __syncthreads();
        const int p = s_p;
        if (p != c) {
            if (r == p)
#pragma unroll
                for (int j = 0; j < NB; ++j) xa[j] = row[j];
            if (r == c)
#pragma unroll
                for (int j = 0; j < NB; ++j) xb[j] = row[j];
        }
        __syncthreads();
        if (p != c) {
            if (r == c)
#pragma unroll
                for (int j = 0; j < NB; ++j) row[j] = xa[j];
            if (r == p)
#pragma unroll
                for (int j = 0; j < NB; ++j) row[j] = xb[j];
        }
        if (r == c) {
            if (zis0(row[kk])) bad = true;
            const z pinv = zrcp(row[kk]);
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                row[j] = (j == kk) ? pinv : zmul(row[j], pinv);
                prow[j] = row[j];
            }
            g.ipiv[c] = p;
        }
        __syncthreads();
        if (own && r != c) {
            const z f = row[kk];
#pragma unroll
            for (int j = 0; j < NB; ++j)
                if (j != kk) zfms(row[j], f, prow[j]);
            row[kk] = zneg(zmul(f, prow[kk]));
        }
    }
    if (own) {
#pragma unroll
        for (int kk = 0; kk < NB; ++kk) {
            if (kk >= nbk) break;
            g.A[r + (long long)(k0 + kk) * g.ld] = row[kk];
        }
    }
    if (bad) atomicOr(status, 1);
}

// exchange rows of every non-panel column and copy the panel rows into Z (nbk x (m - nbk))
__global__ void gj_swapcopy_kernel(const GJDesc* __restrict__ descs, int m, int k0, int nbk) {
    const GJDesc g = descs[blockIdx.y];
    const int jl = blockIdx.x * blockDim.x + threadIdx.x;
    if (jl >= m - nbk) return;
    const int col = jl < k0 ? jl : jl + nbk;
    z* a = g.A + (long long)col * g.ld;
    for (int kk = 0; kk < nbk; ++kk) {
        const int c = k0 + kk;
        const int p = g.ipiv[c];
        if (p != c) {
            const z t = a[c];
            a[c] = a[p];
            a[p] = t;
        }
    }
    for (int kk = 0; kk < nbk; ++kk) g.Zb[kk + (long long)jl * nbk] = a[k0 + kk];
}

template <int BM, int BN, int TM, int TN, int BK>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), 1)
gj_update_kernel(const GJDesc* __restrict__ descs, int m, int k0, int nbk) {
    __shared__ GemmDesc sd;
    if (threadIdx.x == 0) {
        const GJDesc g = descs[blockIdx.y];
        sd.A = zview(g.A + (long long)k0 * g.ld, g.ld);   // the panel columns hold W
        sd.B = zview(g.Zb, nbk);
        sd.C = zview(g.A, g.ld);
        sd.C.cs = k0;
        sd.C.cl = nbk;
        sd.D = zout(g.A, g.ld);
        sd.D.cs = k0;
        sd.D.cl = nbk;
        sd.alpha = zmk(1.0, 0.0);
        sd.beta = zmk(1.0, 0.0);
        sd.m = m;
        sd.n = m - nbk;
        sd.k = nbk;
        sd.nobeta_r0 = k0;          // panel rows are overwritten with W_P Z
        sd.nobeta_r1 = k0 + nbk;
        sd.pad = 0;
    }
    __syncthreads();
    zgemm_tile<BM, BN, TM, TN, BK>(sd, blockIdx.x);
}

__global__ void gj_unscramble_kernel(const GJDesc* __restrict__ descs, int m) {
    const GJDesc g = descs[blockIdx.y];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    for (int k = m - 1; k >= 0; --k) {
        const int p = g.ipiv[k];
        if (p != k) {
            const z t = g.A[r + (long long)k * g.ld];
            g.A[r + (long long)k * g.ld] = g.A[r + (long long)p * g.ld];
            g.A[r + (long long)p * g.ld] = t;
        }
    }
}

template <int NB, int MAXT>
static cudaError_t gj_blocked(const GJDesc* d, int count, int m, int* st, cudaStream_t s) {
    const int threads = ((m + 31) / 32) * 32;
    if (threads > MAXT) return cudaErrorInvalidValue;
    for (int k0 = 0; k0 < m; k0 += NB) {
        const int nbk = (m - k0) < NB ? (m - k0) : NB;
        gj_panel_kernel<NB, MAXT><<<count, threads, 0, s>>>(d, m, k0, nbk, st);
        note_launch();
        const int rest = m - nbk;
        if (rest > 0) {
            gj_swapcopy_kernel<<<dim3((rest + 127) / 128, count), 128, 0, s>>>(d, m, k0, nbk);
            note_launch();
            constexpr int BM = 64, BN = 64, TM = 4, TN = 4, BK = 8;
            const int tiles = ((m + BM - 1) / BM) * ((rest + BN - 1) / BN);
            gj_update_kernel<BM, BN, TM, TN, BK><<<dim3(tiles, count), (BM / TM) * (BN / TN), 0, s>>>(
                d, m, k0, nbk);
            note_launch();
        }
    }
    gj_unscramble_kernel<<<dim3((m + 127) / 128, count), 128, 0, s>>>(d, m);
    note_launch();
    return cudaGetLastError();
}

cudaError_t gj_invert_batch(const GJDesc* d_desc, int count, int m, int* d_status, cudaStream_t s) {
    if (count <= 0 || m <= 0) return cudaSuccess;
    if (m <= GJ_SMALL_MAX) {
        const size_t sh = (size_t)m * m * sizeof(z);
        static bool attr = false;
        if (!attr) {
            cudaError_t e = cudaFuncSetAttribute(gj_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)(GJ_SMALL_MAX * GJ_SMALL_MAX * sizeof(z)));
            if (e != cudaSuccess) return e;
            attr = true;
        }
        gj_small_kernel<<<count, 256, sh, s>>>(d_desc, m, d_status);
        note_launch();
        return cudaGetLastError();
    }
    if (m <= 256) return gj_blocked<16, 256>(d_desc, count, m, d_status, s);
    if (m <= 512) return gj_blocked<8, 512>(d_desc, count, m, d_status, s);
    if (m <= 1024) return gj_blocked<8, 1024>(d_desc, count, m, d_status, s);
    return cudaErrorInvalidValue;
}

}  // namespace rb
