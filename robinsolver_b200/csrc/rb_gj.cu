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
//   2. gj_apply: for every other column, applies the panel's row exchanges and then
//      A[i, rest] += W[i,:] Z for rows outside the panel and A[P, rest] = W_P Z for the panel
//      rows, Z = A[P, rest] after the exchanges.  (Writing the panel rows as Z + (W_P - I) Z
//      instead cancels catastrophically: W_P's diagonal holds the reciprocal pivots, ~h^2 for
//      the FD matrices here.)
// After the last panel the column exchanges are undone in reverse order (gj_unscramble).
#include "rb_gemm_tile.cuh"
#include "rb_kernels.h"

namespace rb {

int gj_panel_width(int m) {
    if (m <= GJ_SMALL_MAX) return 0;
    if (m <= 512) return 16;
    return 8;
}

long long gj_workspace_elems(int m) { return 0; }

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
    // two block barriers per column: (1) per-warp pivot candidates, (2) the scaled pivot row and
    // the displaced row.  Every warp reduces the 32 candidates itself, so the pivot index needs no
    // extra barrier; the holder of the pivot row publishes it already scaled, the holder of row c
    // publishes its row, and after barrier (2) row c takes the pivot row while the pivot's old
    // row takes row c's values and is eliminated like any other row.
    __shared__ z xb[2][NB], prow[2][NB];
    __shared__ double wv[2][32];
    __shared__ int wi[2][32];
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
        const int sb = kk & 1;           // alternate buffers so that barrier (1) of the next column
                                         // also orders this column's reads of prow/xb
        double v = (own && r >= c) ? zabs1(row[kk]) : -1.0;
        int idx = own ? r : 0x7fffffff;
        argmax_warp(v, idx);
        if (lane == 0) { wv[sb][warp] = v; wi[sb][warp] = idx; }
        __syncthreads();                                   // (1)
        v = lane < nwarps ? wv[sb][lane] : -1.0;
        idx = lane < nwarps ? wi[sb][lane] : 0x7fffffff;
        argmax_warp(v, idx);
        const int p = __shfl_sync(0xffffffffu, idx, 0);
        if (r == p) {
            if (zis0(row[kk])) bad = true;
            const z pinv = zrcp(row[kk]);
#pragma unroll
            for (int j = 0; j < NB; ++j) prow[sb][j] = (j == kk) ? pinv : zmul(row[j], pinv);
            g.ipiv[c] = p;
        }
        if (r == c && p != c) {
#pragma unroll
            for (int j = 0; j < NB; ++j) xb[sb][j] = row[j];
        }
        __syncthreads();                                   // (2)
        if (r == c) {
#pragma unroll
            for (int j = 0; j < NB; ++j) row[j] = prow[sb][j];
        } else if (own) {
            if (r == p) {
#pragma unroll
                for (int j = 0; j < NB; ++j) row[j] = xb[sb][j];
            }
            const z f = row[kk];
#pragma unroll
            for (int j = 0; j < NB; ++j)
                if (j != kk) zfms(row[j], f, prow[sb][j]);
            row[kk] = zneg(zmul(f, prow[sb][kk]));
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

// Applies one panel to the other columns: CW whole columns per CTA are staged in shared memory,
// the panel's row exchanges are applied there, and the CTA writes
//     A[i, j] + W[i,:] Z[:, j]   for rows i outside the panel,   W[i,:] Z[:, j]   for panel rows,
// with Z = the (exchanged) panel rows of its own columns and W = the panel columns of A.  A CTA
// owns whole columns, so no other CTA reads what it overwrites.
template <int CW, int NBMAX>
__global__ void __launch_bounds__(256) gj_apply_kernel(const GJDesc* __restrict__ descs, int m, int k0, int nbk) {
    extern __shared__ z cols[];                 // m x CW, column-major (ld m)
    const GJDesc g = descs[blockIdx.y];
    const int rest = m - nbk;
    const int j0 = blockIdx.x * CW;
    const int ncol = min(CW, rest - j0);
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < m * ncol; e += nt) {
        const int r = e % m, q = e / m;
        const int jl = j0 + q;
        const int col = jl < k0 ? jl : jl + nbk;
        cols[r + q * m] = g.A[r + (long long)col * g.ld];
    }
    __syncthreads();
    // the panel's exchanges, in order (each thread owns columns)
    if (tid < ncol)
        for (int kk = 0; kk < nbk; ++kk) {
            const int c = k0 + kk, p = g.ipiv[c];
            if (p != c) {
                const z t = cols[c + tid * m];
                cols[c + tid * m] = cols[p + tid * m];
                cols[p + tid * m] = t;
            }
        }
    __syncthreads();
    for (int r = tid; r < m; r += nt) {
        z w[NBMAX];
#pragma unroll
        for (int kk = 0; kk < NBMAX; ++kk)
            w[kk] = kk < nbk ? g.A[r + (long long)(k0 + kk) * g.ld] : zmk(0.0, 0.0);
        const bool in_panel = r >= k0 && r < k0 + nbk;
        for (int q = 0; q < ncol; ++q) {
            z v = in_panel ? zmk(0.0, 0.0) : cols[r + q * m];
#pragma unroll
            for (int kk = 0; kk < NBMAX; ++kk)
                if (kk < nbk) zfma(v, w[kk], cols[k0 + kk + q * m]);
            const int jl = j0 + q;
            const int col = jl < k0 ? jl : jl + nbk;
            g.A[r + (long long)col * g.ld] = v;
        }
    }
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
    constexpr int CW = 8;
    const size_t sh = (size_t)m * CW * sizeof(z);
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(gj_apply_kernel<CW, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)(1024 * CW * sizeof(z)));
        if (e != cudaSuccess) return e;
        attr = true;
    }
    for (int k0 = 0; k0 < m; k0 += NB) {
        const int nbk = (m - k0) < NB ? (m - k0) : NB;
        gj_panel_kernel<NB, MAXT><<<count, threads, 0, s>>>(d, m, k0, nbk, st);
        note_launch();
        const int rest = m - nbk;
        if (rest > 0) {
            gj_apply_kernel<CW, NB><<<dim3((rest + CW - 1) / CW, count), 256, sh, s>>>(d, m, k0, nbk);
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
    if (m <= 512) return gj_blocked<16, 512>(d_desc, count, m, d_status, s);
    if (m <= 1024) return gj_blocked<8, 1024>(d_desc, count, m, d_status, s);
    return cudaErrorInvalidValue;
}

}  // namespace rb
