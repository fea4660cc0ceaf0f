// rb_gj.cu -- batched in-place Gauss-Jordan inversion of complex128 matrices for sm_100a.
//
// The reference forms inv(D) explicitly (zgetri after zgetrf, robin_tree_module.f90:449-455)
// and applies D and S through their LU factors.  Here every dense inverse the factor/solve
// needs (the leaf's interior Schur complement, D and S of each merge) is formed explicitly by
// Gauss-Jordan elimination with partial pivoting, so that later applications are GEMMs.
// Pivots are chosen as LAPACK's izamax does: largest |re|+|im| in the column, first on ties.
//
// m <= 32: one CTA per matrix holds the whole matrix in shared memory (gj_small).
// m  > 32: blocked Gauss-Jordan by panels of nb = 8 columns.  Per panel:
//   1. elimination of the panel: the pivot search below the diagonal, row exchange, scaling and
//      elimination of every other row, leaving the accumulated transform W in the panel columns;
//   2. update of every other column: the panel's row exchanges, then
//      A[i, rest] += W[i,:] Z for rows outside the panel and A[P, rest] = W_P Z for the panel
//      rows, Z = A[P, rest] after the exchanges.  (Writing the panel rows as Z + (W_P - I) Z
//      instead cancels catastrophically: W_P's diagonal holds the reciprocal pivots, ~h^2 for
//      the FD matrices here.)
//   The resident kernel (gj_resident) runs the whole batch in one cooperative launch with the
//   columns held in shared memory; gj_panel + gj_apply, two launches per panel, are the same
//   arithmetic in the same order, used when the batch does not fit on the device at once.
// After the last panel the column exchanges are undone in reverse order (gj_unscramble).
#include <cstdlib>
#include "rb_gemm_tile.cuh"
#include "rb_kernels.h"

namespace rb {

int gj_panel_width(int m) {
    if (m < GJ_BLOCKED_MIN) return 0;
    return 8;
}

// one complex element per matrix: the resident path's two flag words
long long gj_workspace_elems(int m) { return m < GJ_BLOCKED_MIN ? 0 : 1; }

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

// ---------------------------------------------------------------------------------------------------
// Resident Gauss-Jordan: the whole batch in one launch.  Matrix i is split over P CTAs by whole
// panels of NB columns; CTA j keeps its ppc panels (m x cw complex, cw <= ppc*NB) in shared
// memory for the whole inversion.  The owner of panel p eliminates it (one row per thread in
// registers, as gj_panel_kernel), writes the accumulated transform W_p to the matrix's own
// global storage at panel p's columns (unused while the columns live in shared memory) and its
// pivots to ipiv, and publishes p+1 in the matrix's flag word.  Every CTA then applies step p
// (the exchanges, then A += W_p Z outside the panel rows and W_p Z on them) to its resident
// columns.  The owner of panel p+1 applies step p to that panel first, eliminates and publishes
// it, and only then updates its other columns, so the dependent chain per step is one flag
// hand-off, one panel update and one panel elimination.  After the last step a per-matrix
// counter holds every CTA until all have stopped reading W slots; then the columns go back.
//
// The launch is cooperative (all CTAs co-resident), and every wait is bounded in time: a CTA
// that waits longer than GJ_WAIT_NS sets bit 2 of the status word and returns.
constexpr unsigned long long GJ_WAIT_NS = 1000000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// thread 0 waits until *flag >= target; the outcome is returned to every thread of the CTA
__device__ bool cta_wait_geq(const int* flag, int target, int* status, int* s_ok) {
    if (threadIdx.x == 0) {
        int ok = 1;
        if (ld_acquire_gpu(flag) < target) {
            const unsigned long long t0 = global_ns();
            int spins = 0;
            while (ld_acquire_gpu(flag) < target) {
                if (++spins > 32) __nanosleep(40);
                if (global_ns() - t0 > GJ_WAIT_NS) {
                    ok = 0;
                    atomicOr(status, 2);
                    break;
                }
            }
        }
        *s_ok = ok;
    }
    __syncthreads();
    const bool ok = *s_ok != 0;
    __syncthreads();                     // s_ok may be rewritten by the next wait
    return ok;
}

// Slots of one elimination column, double-buffered by column parity: column kk writes set kk & 1,
// so a column's slots are rewritten two columns later, after every thread has passed the block
// barrier that follows its last read of them -- one barrier per column fewer than single slots.
template <int NB>
struct ResShared {
    z xb[2][NB], prow[2][NB];
    unsigned kh[2][32], kl[2][32];
    int ki[2][32];
    int spv[NB];                         // pivots of the step being applied
    int ok;
};

// warp argmax over (hi, lo) = the bit pattern of a non-negative double (which orders like the
// value), ties to the smaller row: three warp reductions instead of a shuffle tree
__device__ __forceinline__ void warp_key_max(unsigned& hi, unsigned& lo, int& id) {
    const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
    const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
    id = __reduce_min_sync(0xffffffffu, (hi == mh && lo == ml) ? id : 0x7fffffff);
    hi = mh;
    lo = ml;
}

// CTA-wide argmax of v over the valid rows (largest first, then smallest row), in slot set b:
// one block barrier; every thread gets the row
template <int NB>
__device__ __forceinline__ int block_argmax(double v, bool valid, int r, ResShared<NB>& sh, int b) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
    unsigned hi = valid ? (unsigned)__double2hiint(v) : 0u;
    unsigned lo = valid ? (unsigned)__double2loint(v) : 0u;
    int id = valid ? r : 0x7fffffff;
    warp_key_max(hi, lo, id);
    if (lane == 0) {
        sh.kh[b][warp] = hi;
        sh.kl[b][warp] = lo;
        sh.ki[b][warp] = id;
    }
    __syncthreads();
    hi = lane < nwarps ? sh.kh[b][lane] : 0u;
    lo = lane < nwarps ? sh.kl[b][lane] : 0u;
    id = lane < nwarps ? sh.ki[b][lane] : 0x7fffffff;
    warp_key_max(hi, lo, id);
    return id;
}

// Eliminates a panel of nbk columns (matrix columns k0..) whose current values are in row[][]:
// RPT rows per thread (rows tid + i*blockDim.x), two block barriers per column (pivot candidates;
// scaled pivot row and displaced row).  On return row[][] holds the panel's transform W and the
// pivots are in ipiv.
template <int NB, int RPT>
__device__ __forceinline__ void res_eliminate_regs(z (&row)[RPT][NB], int m, int k0, int nbk, int* ipiv, int* status,
                                                   ResShared<NB>& sh) {
    const int tid = threadIdx.x, nt = blockDim.x;
    bool bad = false;
#pragma unroll
    for (int kk = 0; kk < NB; ++kk) {
        if (kk >= nbk) break;
        const int c = k0 + kk, b = kk & 1;
        // this thread's candidate: its largest entry on or below row c, first on ties
        double v = 0.0;
        int vr = -1;
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            const int r = tid + i * nt;
            const double a = zabs1(row[i][kk]);
            if (r < m && r >= c && (vr < 0 || a > v)) { v = a; vr = r; }
        }
        const int p = block_argmax<NB>(v, vr >= 0, vr, sh, b);
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            const int r = tid + i * nt;
            if (r == p) {
                if (zis0(row[i][kk])) bad = true;
                const z pinv = zrcp(row[i][kk]);
#pragma unroll
                for (int j = 0; j < NB; ++j) sh.prow[b][j] = (j == kk) ? pinv : zmul(row[i][j], pinv);
                ipiv[c] = p;
            }
            if (r == c && p != c) {
#pragma unroll
                for (int j = 0; j < NB; ++j) sh.xb[b][j] = row[i][j];
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            const int r = tid + i * nt;
            if (r == c) {
#pragma unroll
                for (int j = 0; j < NB; ++j) row[i][j] = sh.prow[b][j];
            } else if (r < m) {
                if (r == p) {
#pragma unroll
                    for (int j = 0; j < NB; ++j) row[i][j] = sh.xb[b][j];
                }
                const z f = row[i][kk];
#pragma unroll
                for (int j = 0; j < NB; ++j)
                    if (j != kk) zfms(row[i][j], f, sh.prow[b][j]);
                row[i][kk] = zneg(zmul(f, sh.prow[b][kk]));
            }
        }
    }
    if (bad) atomicOr(status, 1);
}

// Stores an eliminated panel: W to the local columns [q0, q0+nbk) and to Wg (ld wld), then a
// block barrier.
template <int NB, int RPT>
__device__ __forceinline__ void res_store_panel(const z (&row)[RPT][NB], z* cols, int m, int q0, int nbk, z* Wg,
                                                long long wld) {
    const int tid = threadIdx.x, nt = blockDim.x;
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int r = tid + i * nt;
        if (r >= m) continue;
#pragma unroll
        for (int kk = 0; kk < NB; ++kk) {
            if (kk >= nbk) break;
            cols[r + (q0 + kk) * m] = row[i][kk];
            Wg[r + (long long)kk * wld] = row[i][kk];
        }
    }
    __syncthreads();
}

// Eliminates the panel held at local columns [q0, q0+nbk) (matrix columns k0..) and stores it.
template <int NB, int RPT>
__device__ __noinline__ void res_eliminate(z* cols, int m, int q0, int k0, int nbk, z* Wg, long long wld, int* ipiv,
                                           int* status, ResShared<NB>& sh) {
    const int tid = threadIdx.x, nt = blockDim.x;
    z row[RPT][NB];
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int r = tid + i * nt;
#pragma unroll
        for (int kk = 0; kk < NB; ++kk) row[i][kk] = (r < m && kk < nbk) ? cols[r + (q0 + kk) * m] : zmk(0.0, 0.0);
    }
    res_eliminate_regs<NB, RPT>(row, m, k0, nbk, ipiv, status, sh);
    res_store_panel<NB, RPT>(row, cols, m, q0, nbk, Wg, wld);
}

// Applies step (panel at matrix columns k0.., nbk wide, pivots at piv (shared memory), W at W with
// ld wld, read through L2 when w_global) to the local columns [qa, qb) except [xa, xb).  The panel's row
// exchanges move only the panel rows and the pivot rows below the panel; their exchanged values
// (row a takes stored row src(a), src = the transpositions traced backwards) are gathered in
// parallel into zs (2*NB slots per column: slot t < NB panel row k0+t, slot NB+t pivot row t
// unless it repeats), the displaced pivot rows are written back, and then every thread updates
// its rows: A + W Z outside the panel rows, W_P Z on them, Z = the gathered panel rows.  Same
// operations, in the same order, as exchanging row by row and then updating.
template <int NB, int RPT>
__device__ __noinline__ void res_apply(z* cols, z* zs, int m, int k0, int nbk, const z* W, long long wld,
                                       bool w_global, const int* piv, int qa, int qb, int xa, int xb) {
    if (qb <= qa) return;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int nq = qb - qa;
    {
        int pv[NB];
#pragma unroll
        for (int kk = 0; kk < NB; ++kk) pv[kk] = kk < nbk ? piv[kk] : -1;
        for (int e = tid; e < 2 * NB * nq; e += nt) {
            const int t = e % (2 * NB), q = qa + e / (2 * NB);
            if (q >= xa && q < xb) continue;
            int a = -1;
            if (t < nbk) {
                a = k0 + t;
            } else if (t >= NB && t - NB < nbk) {
                int pt = -1;
#pragma unroll
                for (int u = 0; u < NB; ++u)
                    if (u == t - NB) pt = pv[u];
                bool dup = pt < k0 + nbk;
#pragma unroll
                for (int u = 0; u < NB; ++u)
                    if (u < t - NB && pv[u] == pt) dup = true;
                if (!dup) a = pt;
            }
            if (a < 0) continue;
            int jr = a;
#pragma unroll
            for (int kk = NB - 1; kk >= 0; --kk) {
                const int c = k0 + kk;
                if (kk < nbk) jr = (jr == c) ? pv[kk] : (jr == pv[kk] ? c : jr);
            }
            zs[t + (q - qa) * 2 * NB] = cols[jr + q * m];
        }
        __syncthreads();
        for (int e = tid; e < NB * nq; e += nt) {
            const int t = e % NB, q = qa + e / NB;
            if ((q >= xa && q < xb) || t >= nbk) continue;
            int pt = -1;
#pragma unroll
            for (int u = 0; u < NB; ++u)
                if (u == t) pt = pv[u];
            bool dup = pt < k0 + nbk;
#pragma unroll
            for (int u = 0; u < NB; ++u)
                if (u < t && pv[u] == pt) dup = true;
            if (!dup) cols[pt + q * m] = zs[NB + t + (q - qa) * 2 * NB];
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int r = tid + i * nt;
        if (r >= m) continue;
        z w[NB];
#pragma unroll
        for (int kk = 0; kk < NB; ++kk)
            w[kk] = kk < nbk ? (w_global ? __ldcg(W + r + kk * wld) : W[r + kk * wld]) : zmk(0.0, 0.0);
        const bool in_panel = r >= k0 && r < k0 + nbk;
        for (int q = qa; q < qb; ++q) {
            if (q >= xa && q < xb) continue;
            z v = in_panel ? zmk(0.0, 0.0) : cols[r + q * m];
            const z* zq = zs + (q - qa) * 2 * NB;
#pragma unroll
            for (int kk = 0; kk < NB; ++kk)
                if (kk < nbk) zfma(v, w[kk], zq[kk]);
            cols[r + q * m] = v;
        }
    }
    __syncthreads();
}

template <int NB, int MAXT, int RPT>
__global__ void __launch_bounds__(MAXT, MAXT <= 256 ? 512 / MAXT : 1) gj_resident_kernel(
    const GJDesc* __restrict__ descs, int m, int npanels, int ppc, int P, int* status) {
    extern __shared__ z sm[];
    __shared__ ResShared<NB> sh;
    const int mat = blockIdx.x / P, j = blockIdx.x % P;
    const GJDesc g = descs[mat];
    const int pa = j * ppc, pb = min(npanels, pa + ppc);
    const int c0 = pa * NB, cw = min(m, pb * NB) - c0;
    z* cols = sm;                                   // m x cw, column-major (ld m)
    z* zs = sm + (size_t)m * ppc * NB;              // 2NB x cw: exchanged panel and pivot rows
    int* pub = reinterpret_cast<int*>(g.Zb);        // panels published
    int* done = pub + 1;                            // CTAs past their last step
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < m * cw; e += nt) {
        const int r = e % m, q = e / m;
        cols[r + q * m] = __ldcg(g.A + r + (long long)(c0 + q) * g.ld);
    }
    __syncthreads();
    auto publish = [&](int p) {          // res_eliminate ended with a block barrier
        if (tid == 0) {
            __threadfence();
            st_release_gpu(pub, p + 1);
        }
    };
    if (pa == 0) {
        res_eliminate<NB, RPT>(cols, m, 0, 0, min(NB, m), g.A, g.ld, g.ipiv, status, sh);
        publish(0);
    }
    for (int p = 0; p < npanels; ++p) {
        const int k0 = p * NB, nbk = min(NB, m - k0);
        const bool own = p >= pa && p < pb;
        if (!own && !cta_wait_geq(pub, p + 1, status, &sh.ok)) return;
        // the step's pivots, read once by the CTA: read by every thread, the same 32 bytes made an
        // L2 hot spot of thousands of requests per step that cost the chain ~2.5 us a panel
        if (tid < NB) sh.spv[tid] = tid < nbk ? __ldcg(g.ipiv + k0 + tid) : -1;
        __syncthreads();
        const z* W = own ? cols + (size_t)(k0 - c0) * m : g.A + (long long)k0 * g.ld;
        const long long wld = own ? m : g.ld;
        const int* piv = sh.spv;
        const int xa = own ? k0 - c0 : 0, xb = own ? k0 - c0 + nbk : 0;
        const int nx = p + 1;
        if (nx < npanels && nx >= pa && nx < pb) {
            const int qn = nx * NB - c0, nbn = min(NB, m - nx * NB);
            res_apply<NB, RPT>(cols, zs, m, k0, nbk, W, wld, !own, piv, qn, qn + nbn, xa, xb);
            res_eliminate<NB, RPT>(cols, m, qn, nx * NB, nbn, g.A + (long long)nx * NB * g.ld, g.ld, g.ipiv, status,
                                   sh);
            publish(nx);
            res_apply<NB, RPT>(cols, zs, m, k0, nbk, W, wld, !own, piv, 0, qn, xa, xb);
            res_apply<NB, RPT>(cols, zs, m, k0, nbk, W, wld, !own, piv, qn + nbn, cw, xa, xb);
        } else {
            res_apply<NB, RPT>(cols, zs, m, k0, nbk, W, wld, !own, piv, 0, cw, xa, xb);
        }
    }
    // no CTA of this matrix reads a W slot any more once all have arrived here
    if (tid == 0) {
        __threadfence();
        atomicAdd(done, 1);
    }
    if (!cta_wait_geq(done, P, status, &sh.ok)) return;
    for (int e = tid; e < m * cw; e += nt) {
        const int r = e % m, q = e / m;
        g.A[r + (long long)(c0 + q) * g.ld] = cols[r + q * m];
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
    static DeviceAttrCache attr;
    {
        cudaError_t e = ensure_smem_attr(gj_apply_kernel<CW, NB>, 1024 * CW * sizeof(z), attr);
        if (e != cudaSuccess) return e;
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

// Resident path: the smallest number of panels per CTA whose grid is co-resident; false when
// even one CTA per panel group cannot hold the batch (the caller then runs the blocked path).
template <int NB, int MAXT, int RPT>
static cudaError_t gj_resident(const GJDesc* d, int count, int m, void* flags, int* st, cudaStream_t s, bool* done) {
    *done = false;
    const int threads = ((m + RPT - 1) / RPT + 31) / 32 * 32;
    if (threads > MAXT) return cudaSuccess;
    const int npanels = (m + NB - 1) / NB;
    int dev = 0, nsm = 0, coop = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev)) != cudaSuccess) return e;
    if (!coop) return cudaSuccess;
    constexpr int SMEM_MAX = 227 * 1024;
    static DeviceAttrCache attr;
    e = ensure_smem_attr(gj_resident_kernel<NB, MAXT, RPT>, SMEM_MAX - sizeof(ResShared<NB>), attr);
    if (e != cudaSuccess) return e;
    // fewest panels per CTA: a CTA that owns more panels updates its others before it can
    // eliminate its next one, which lengthens the chain (1024^2, L=12: 25.5 ms factor with one
    // panel per CTA, 26.9 with at least two, 29.3 with at least six)
    for (int ppc = 1; ppc <= npanels; ++ppc) {
        const int P = (npanels + ppc - 1) / ppc;
        const size_t sh = ((size_t)m + 2 * NB) * ppc * NB * sizeof(z);
        if (sh + sizeof(ResShared<NB>) > (size_t)SMEM_MAX) break;
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gj_resident_kernel<NB, MAXT, RPT>, threads, sh);
        if (e != cudaSuccess) return e;
        if ((long long)count * P > (long long)per_sm * nsm) continue;
        if ((e = cudaMemsetAsync(flags, 0, (size_t)count * sizeof(z), s)) != cudaSuccess) return e;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(count * P));
        cfg.blockDim = dim3((unsigned)threads);
        cfg.dynamicSmemBytes = sh;
        cfg.stream = s;
        cudaLaunchAttribute la[1];
        la[0].id = cudaLaunchAttributeCooperative;
        la[0].val.cooperative = 1;
        cfg.attrs = la;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, gj_resident_kernel<NB, MAXT, RPT>, d, m, npanels, ppc, P, st);
        if (e != cudaSuccess) return e;
        note_launch();
        gj_unscramble_kernel<<<dim3((m + 127) / 128, count), 128, 0, s>>>(d, m);
        note_launch();
        *done = true;
        return cudaGetLastError();
    }
    return cudaSuccess;
}

// RB_GJ_RESIDENT=0 selects the blocked path (read at every launch, so that a process can compare)
static bool resident_enabled() {
    const char* v = std::getenv("RB_GJ_RESIDENT");
    return !(v && v[0] == '0');
}

cudaError_t gj_invert_batch(const GJDesc* d_desc, int count, int m, void* work, int* d_status, cudaStream_t s) {
    if (count <= 0 || m <= 0) return cudaSuccess;
    if (m < GJ_BLOCKED_MIN) {
        const size_t sh = (size_t)m * m * sizeof(z);
        static DeviceAttrCache attr;
        {
            cudaError_t e = ensure_smem_attr(gj_small_kernel, GJ_SMALL_MAX * GJ_SMALL_MAX * sizeof(z), attr);
            if (e != cudaSuccess) return e;
        }
        gj_small_kernel<<<count, 256, sh, s>>>(d_desc, m, d_status);
        note_launch();
        return cudaGetLastError();
    }
    if (resident_enabled() && work) {
        bool done = false;
        cudaError_t e = cudaSuccess;
        if (m <= 64) e = gj_resident<8, 64, 1>(d_desc, count, m, work, d_status, s, &done);
        else if (m <= 128) e = gj_resident<8, 128, 1>(d_desc, count, m, work, d_status, s, &done);
        else if (m <= 256) e = gj_resident<8, 256, 1>(d_desc, count, m, work, d_status, s, &done);
        else if (m <= 512) e = gj_resident<8, 512, 1>(d_desc, count, m, work, d_status, s, &done);
        else if (m <= 1024) e = gj_resident<8, 512, 2>(d_desc, count, m, work, d_status, s, &done);
        if (e != cudaSuccess || done) return e;
    }
    if (m <= 64) return gj_blocked<8, 64>(d_desc, count, m, d_status, s);
    if (m <= 256) return gj_blocked<8, 256>(d_desc, count, m, d_status, s);
    if (m <= 512) return gj_blocked<8, 512>(d_desc, count, m, d_status, s);
    if (m <= 1024) return gj_blocked<8, 1024>(d_desc, count, m, d_status, s);
    return cudaErrorInvalidValue;
}

}  // namespace rb
