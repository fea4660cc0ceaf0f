// rb_leaf.cu -- structured leaf factor and leaf solve for sm_100a (one CTA per leaf).
//
// Leaf algebra.  The reference's leaf matrix A (FD_matrix_row, fd_module.f90:104-224) has its rows/
// columns in lin2fgrid order: the nb = 2(a+b) cornerless boundary points first (faces
// x1 x2 y1 y2), then the a*b interior points x-fastest.  Every boundary row r reads only
// itself and two interior points along the inward normal:
//     A(r,r) = i*kb + (8/3)/h,  A(r,p1) = -3/h,  A(r,p2) = (1/3)/h        (fd_module.f90:207-215)
// so A_bb is diagonal and the boundary unknowns condense exactly.  With
// d_r = A(r,r), c1 = -3/h, c2 = 1/(3h) and w_c = (8/3)/h^2 (the interior row next to boundary
// point c couples to it with that weight, fd_module.f90:150-153):
//     S      = A_ii - A_ib A_bb^-1 A_bi                       (a*b x a*b)
//     A^-1   = [[ (I - A_bi A^-1_ib) / d ,  -A_bi S^-1 / d ],
//               [ -S^-1 A_ib / d          ,   S^-1          ]]
// The reference's leaf Robin-to-Robin map is R X with X = A^-1 [I; 0] and R the outgoing rows
// sigma*u + tau*(8/3 u - 3 u_p1 + 1/3 u_p2)/h, sigma = -i*kb, tau = 1
// (RTR_update, robin_tree_module.f90:683-713).  Row r of Y = R A^-1 is
//     Y(r,:) = (sigma'_r / d_r) e_r + (2 i kb / d_r) (c1 A^-1(p1,:) + c2 A^-1(p2,:)),
// sigma'_r = sigma + (8/3)/h, because sigma'_r - d_r = -2 i kb.  Y(:, 0:nb) is the leaf RtR,
// Y(:, nb:n) maps an interior source to the outgoing data of the particular solution
// (fd_leaf_solve + fd_outgoing_bc, fd_module.f90:390-513).
//
// The condensed interior operator S inherits the 5-point stencil of FD_matrix_row
// (fd_module.f90:140-181): with the interior points ordered x-fastest (igrid2lin, fd_module.f90:835-841) it is block tridiagonal,
// b blocks of a x a,
//     S = tridiag(Lo_j, D_j, Up_j),  D_j tridiagonal,  Lo_j = diag(lam_j),  Up_j = diag(mu_j).
// Block elimination without exchanges between blocks (the blocks are diagonally dominant
// Laplacian blocks shifted by the potential; each block inverse pivots by |re|+|im|):
//     Sig_1 = D_1,  Sig_j = D_j - Lo_j Sig_{j-1}^-1 Up_{j-1},       S = L U,
//     L = [I; Lo_j Sig_{j-1}^-1 below],  U = [Sig_j; Up_j above].
// The leaf factor keeps Sig_j^-1 (b a^2 values instead of the reference's (ab+nb)^2 LU) and
// forms the Robin-to-Robin data Y = R A^-1 from Q = C S^-1, where row r of C is
// c1 e_p1(r) + c2 e_p2(r) (the interior part of the outgoing row of RTR_update,
// robin_tree_module.f90:699-713): Q^T = S^-T C^T by one block forward and one block backward
// sweep with nb right-hand sides.  Then, by the row formula above,
//     Y(r, nb+s) = f_r Q(r,s),   Y(r,c) = (sigma'_r/d_r) delta_rc - f_r (w_c/d_c) Q(r, p1(c)),
//     f_r = 2 i kb / d_r.
// The leaf solve applies A^-1 [g; f] (fd_leaf_solve + fd_leaf_update, fd_module.f90:390-566)
// through the same block factors: t = f - A_ib A_bb^-1 g, S u_i = t, u_b = (g - A_bi u_i)/d.
#include <cstdlib>
#include <cstring>
#include "rb_gemm_dmma.cuh"   // dmma884
#include "rb_kernels.h"

namespace rb {

__device__ __forceinline__ void leaf_bpoint2(int a, int b, int r, int& axis, int& p1, int& p2) {
    if (r < b) { axis = 0; p1 = r * a; p2 = r * a + 1; }
    else if (r < 2 * b) { const int j = r - b; axis = 0; p1 = j * a + (a - 1); p2 = j * a + (a - 2); }
    else if (r < 2 * b + a) { const int i = r - 2 * b; axis = 1; p1 = i; p2 = a + i; }
    else { const int i = r - 2 * b - a; axis = 1; p1 = (b - 1) * a + i; p2 = (b - 2) * a + i; }
}

__device__ __forceinline__ void stencil1(int i, int a, double& wm, double& w0, double& wp) {
    if (i == 1) { wm = 8.0 / 3.0; w0 = -4.0; wp = 4.0 / 3.0; }
    else if (i == a) { wm = 4.0 / 3.0; w0 = -4.0; wp = 8.0 / 3.0; }
    else { wm = 1.0; w0 = -2.0; wp = 1.0; }
}

// constants of one leaf's condensed stencil
struct LeafConst {
    double hx, hy, hx2, hy2;
    z rdx, rdy;                 // 1 / d for x-face and y-face boundary points
    double c1x, c2x, c1y, c2y;  // -3/h, 1/(3h)
    double wbx, wby;            // (8/3)/h^2
};

__device__ __forceinline__ LeafConst leaf_const(const double* hh, int leaf, double kb) {
    LeafConst c;
    c.hx = hh[2 * leaf];
    c.hy = hh[2 * leaf + 1];
    c.hx2 = c.hx * c.hx;
    c.hy2 = c.hy * c.hy;
    c.rdx = zrcp(zmk((8.0 / 3.0) / c.hx, kb));
    c.rdy = zrcp(zmk((8.0 / 3.0) / c.hy, kb));
    c.c1x = -3.0 / c.hx; c.c2x = (1.0 / 3.0) / c.hx;
    c.c1y = -3.0 / c.hy; c.c2y = (1.0 / 3.0) / c.hy;
    c.wbx = (8.0 / 3.0) / c.hx2;
    c.wby = (8.0 / 3.0) / c.hy2;
    return c;
}

// entry (r, c) of the diagonal block D_j (grid row jj = j+1) of S
__device__ __forceinline__ z block_d(const LeafConst& L, int a, int b, int jj, int r, int c, z k) {
    const int i = r + 1;
    double wxm, wx0, wxp, wym, wy0, wyp;
    stencil1(i, a, wxm, wx0, wxp);
    stencil1(jj, b, wym, wy0, wyp);
    z v = zmk(0.0, 0.0);
    if (c == r) {
        v = zmk((k.x + wx0 / L.hx2) + wy0 / L.hy2, k.y);
        if (i == 1 || i == a) v = zsub(v, zscale(L.wbx * L.c1x, L.rdx));
        if (jj == 1 || jj == b) v = zsub(v, zscale(L.wby * L.c1y, L.rdy));
    } else if (c == r + 1 && i < a) {
        v = zmk(wxp / L.hx2, 0.0);
        if (i == 1) v = zsub(v, zscale(L.wbx * L.c2x, L.rdx));
    } else if (c == r - 1 && i > 1) {
        v = zmk(wxm / L.hx2, 0.0);
        if (i == a) v = zsub(v, zscale(L.wbx * L.c2x, L.rdx));
    }
    return v;
}
// Lo_j(i,i) = S(e, e-a) for grid row jj >= 2 and Up_j(i,i) = S(e, e+a) for jj <= b-1
__device__ __forceinline__ z block_lo(const LeafConst& L, int b, int jj) {
    double wm, w0, wp;
    stencil1(jj, b, wm, w0, wp);
    z v = zmk(wm / L.hy2, 0.0);
    if (jj == b) v = zsub(v, zscale(L.wby * L.c2y, L.rdy));
    return v;
}
__device__ __forceinline__ z block_up(const LeafConst& L, int b, int jj) {
    double wm, w0, wp;
    stencil1(jj, b, wm, w0, wp);
    z v = zmk(wp / L.hy2, 0.0);
    if (jj == 1) v = zsub(v, zscale(L.wby * L.c2y, L.rdy));
    return v;
}

// In-place Gauss-Jordan inverse of an m x m column-major matrix in shared memory by the whole
// CTA (partial pivoting by |re|+|im|, first maximum).  Returns false on an exactly zero pivot.
__device__ bool cta_gj_invert(z* S, int m, z* fcol, int* ipiv, int* sp) {
    const int tid = threadIdx.x, nt = blockDim.x;
    bool ok = true;
    for (int k = 0; k < m; ++k) {
        if (tid < 32) {
            double best = -1.0;
            int bi = m;
            for (int r = k + tid; r < m; r += 32) {
                const double v = zabs1(S[r + k * m]);
                if (v > best) { best = v; bi = r; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, best, o);
                const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (tid == 0) { *sp = bi; ipiv[k] = bi; }
        }
        __syncthreads();
        const int p = *sp;
        if (p != k)
            for (int c = tid; c < m; c += nt) {
                const z t = S[k + c * m];
                S[k + c * m] = S[p + c * m];
                S[p + c * m] = t;
            }
        __syncthreads();
        const z piv = S[k + k * m];
        if (piv.x == 0.0 && piv.y == 0.0) ok = false;
        const z pinv = zrcp(piv);
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
    return ok;
}

// ---------------------------------------------------------------------------------------------------
// Leaf factor: Sig_j^-1 for every block and Y = R A^-1 (nb x n, ld nb).  Shared memory:
// sig (a^2), sigp (a^2), v0, v1 (a x nb each), fcol (a), ipiv (a), sp.
__global__ void __launch_bounds__(256) leaf_block_factor_kernel(LeafGeom g, const double* __restrict__ hh,
                                                                const z* __restrict__ kv, z* __restrict__ sinv,
                                                                z* __restrict__ Y, int* status) {
    extern __shared__ z sm[];
    const int leaf = blockIdx.x;
    const int a = g.a, b = g.b, nb = g.nb, n = g.n, ab = a * b, aa = a * a;
    const int tid = threadIdx.x, nt = blockDim.x;
    z* sig = sm;
    z* sigp = sig + aa;
    z* v0 = sigp + aa;
    z* v1 = v0 + (size_t)a * nb;
    z* fcol = v1 + (size_t)a * nb;
    int* ipiv = reinterpret_cast<int*>(fcol + a);
    int* sp = ipiv + a;
    const LeafConst L = leaf_const(hh, leaf, g.kb);
    const z* kl = kv + (size_t)leaf * ab;
    z* Sl = sinv + (size_t)leaf * b * aa;
    z* Yl = Y + (size_t)leaf * nb * n;
    bool ok = true;

    // ---- block LU: Sig_j^-1, j = 0..b-1 ------------------------------------------------------
    for (int j = 0; j < b; ++j) {
        const int jj = j + 1;
        const z lam = jj > 1 ? block_lo(L, b, jj) : zmk(0.0, 0.0);
        const z mup = jj > 1 ? block_up(L, b, jj - 1) : zmk(0.0, 0.0);
        for (int e = tid; e < aa; e += nt) {
            const int r = e % a, c = e / a;
            z v = block_d(L, a, b, jj, r, c, kl[j * a + r]);
            if (jj > 1) zfms(v, zmul(lam, mup), sigp[e]);
            sig[e] = v;
        }
        __syncthreads();
        ok &= cta_gj_invert(sig, a, fcol, ipiv, sp);
        for (int e = tid; e < aa; e += nt) {
            Sl[(size_t)j * aa + e] = sig[e];
            sigp[e] = sig[e];
        }
        __syncthreads();
    }

    // ---- forward sweep of S^T Z = C^T: v_j = Sig_j^-T (c_j - Up_{j-1} v_{j-1}) ---------------------
    // v_j (a x nb, ld a) is kept in shared memory and stored transposed into Y(:, nb + j*a + i).
    z* vp = v0;
    z* vc = v1;
    for (int j = 0; j < b; ++j) {
        const int jj = j + 1;
        for (int e = tid; e < aa; e += nt) sig[e] = Sl[(size_t)j * aa + e];
        const z mup = jj > 1 ? block_up(L, b, jj - 1) : zmk(0.0, 0.0);
        __syncthreads();
        for (int e = tid; e < a * nb; e += nt) {
            const int i = e % a, r = e / a;
            int ax, p1, p2;
            leaf_bpoint2(a, b, r, ax, p1, p2);
            const double hr = ax == 0 ? L.hx : L.hy;
            const double c1 = -3.0 / hr, c2 = (1.0 / 3.0) / hr;
            z acc = zmk(0.0, 0.0);
            for (int q = 0; q < a; ++q) {
                const int eq = j * a + q;
                z rhs = zmk((eq == p1 ? c1 : 0.0) + (eq == p2 ? c2 : 0.0), 0.0);
                if (jj > 1) zfms(rhs, mup, vp[q + r * a]);
                zfma(acc, sig[q + i * a], rhs);       // (Sig^-T)(i,q) = Sig^-1(q,i)
            }
            vc[e] = acc;
            Yl[r + (size_t)(nb + j * a + i) * nb] = acc;
        }
        __syncthreads();
        z* t = vp; vp = vc; vc = t;
    }
    // ---- backward sweep: z_{j-1} = v_{j-1} - Sig_{j-1}^-T Lo_j z_j; z_{b-1} = v_{b-1} (in vp) -------
    for (int j = b - 1; j >= 1; --j) {
        const int jj = j + 1;              // grid row of block j
        const z lam = block_lo(L, b, jj);
        for (int e = tid; e < aa; e += nt) sig[e] = Sl[(size_t)(j - 1) * aa + e];
        __syncthreads();
        for (int e = tid; e < a * nb; e += nt) {
            const int i = e % a, r = e / a;
            z acc = Yl[r + (size_t)(nb + (j - 1) * a + i) * nb];
            for (int q = 0; q < a; ++q) zfms(acc, sig[q + i * a], zmul(lam, vp[q + r * a]));
            vc[e] = acc;
            Yl[r + (size_t)(nb + (j - 1) * a + i) * nb] = acc;
        }
        __syncthreads();
        z* t = vp; vp = vc; vc = t;
    }
    __syncthreads();
    // ---- Y = R A^-1 from Q(r, s) = Z(s, r) = Y(r, nb+s) -------------------------------------------
    for (int e = tid; e < nb * nb; e += nt) {
        const int r = e % nb, c = e / nb;
        int ax, p1, p2, axc, p1c, p2c;
        leaf_bpoint2(a, b, r, ax, p1, p2);
        leaf_bpoint2(a, b, c, axc, p1c, p2c);
        const z rd = ax == 0 ? L.rdx : L.rdy;
        const z f = zmul(zmk(0.0, 2.0 * g.kb), rd);
        const z wd = axc == 0 ? zscale(L.wbx, L.rdx) : zscale(L.wby, L.rdy);
        z v = zneg(zmul(zmul(f, wd), Yl[r + (size_t)(nb + p1c) * nb]));
        if (c == r) {
            const double hr = ax == 0 ? L.hx : L.hy;
            v = zadd(v, zmul(zmk((8.0 / 3.0) / hr, -g.kb), rd));
        }
        Yl[e] = v;
    }
    __syncthreads();
    for (int e = tid; e < nb * ab; e += nt) {
        const int r = e % nb;
        int ax, p1, p2;
        leaf_bpoint2(a, b, r, ax, p1, p2);
        const z f = zmul(zmk(0.0, 2.0 * g.kb), ax == 0 ? L.rdx : L.rdy);
        Yl[(size_t)nb * nb + e] = zmul(f, Yl[(size_t)nb * nb + e]);
    }
    if (!ok && tid == 0) atomicOr(status, 1);
}

// ---------------------------------------------------------------------------------------------------
// Warp-per-leaf factor for a = 16 (every leaf of a 16x16 grid): the same algebra as
// leaf_block_factor_kernel with no block barriers.  A 16x16 block lives in registers, lane l
// holding row l%16, columns 8*(l/16)..+7; Gauss-Jordan pivots by shuffles (|re|+|im|, first
// maximum) and the column exchanges are undone through the warp's shared memory.  In the
// S^T Z = C^T sweeps each lane carries one right-hand side (a 16-vector per block) at a time.
__global__ void __launch_bounds__(128) leaf_warp_factor_kernel(LeafGeom g, int nleaves, const double* __restrict__ hh,
                                                               const z* __restrict__ kv, z* __restrict__ sinv,
                                                               z* __restrict__ Y, int* status) {
    constexpr int A = 16, AA = 256;
    __shared__ z wsm[4][AA];
    __shared__ int wpiv[4][2 * A];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int leaf = blockIdx.x * 4 + wib;
    if (leaf >= nleaves) return;
    z* sm = wsm[wib];
    int* piv = wpiv[wib];
    const int b = g.b, nb = g.nb, n = g.n, ab = A * b;
    const LeafConst L = leaf_const(hh, leaf, g.kb);
    const z* kl = kv + (size_t)leaf * ab;
    z* Sl = sinv + (size_t)leaf * b * AA;
    z* Yl = Y + (size_t)leaf * nb * n;
    const int r = lane & 15, hf = lane >> 4;          // row, column half
    z a[8], prev[8];
    bool ok = true;

    // ---- block LU ---------------------------------------------------------------------------------
    for (int j = 0; j < b; ++j) {
        const int jj = j + 1;
        const z lm = jj > 1 ? zmul(block_lo(L, b, jj), block_up(L, b, jj - 1)) : zmk(0.0, 0.0);
        const z kr = kl[j * A + r];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            z v = block_d(L, A, b, jj, r, hf * 8 + e, kr);
            if (jj > 1) zfms(v, lm, prev[e]);
            a[e] = v;
        }
#pragma unroll
        for (int k = 0; k < A; ++k) {
            const int hk = k >> 3, ek = k & 7;
            double mag = (hf == hk && r >= k) ? zabs1(a[ek]) : -1.0;
            int idx = r;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double om = __shfl_xor_sync(0xffffffffu, mag, o);
                const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
                if (om > mag || (om == mag && oi < idx)) { mag = om; idx = oi; }
            }
            const int p = idx;
            if (lane == 0) piv[k] = p;
            if (p != k) {                           // exchange rows k and p
                const int src = (r == k ? p : (r == p ? k : r)) + 16 * hf;
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const double x = __shfl_sync(0xffffffffu, a[e].x, src);
                    const double y = __shfl_sync(0xffffffffu, a[e].y, src);
                    a[e] = zmk(x, y);
                }
            }
            const z pv = zmk(__shfl_sync(0xffffffffu, a[ek].x, k + 16 * hk),
                             __shfl_sync(0xffffffffu, a[ek].y, k + 16 * hk));
            if (pv.x == 0.0 && pv.y == 0.0) ok = false;
            const z pinv = zrcp(pv);
            const z f = zmk(__shfl_sync(0xffffffffu, a[ek].x, r + 16 * hk),
                            __shfl_sync(0xffffffffu, a[ek].y, r + 16 * hk));
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const z pr = zmul(zmk(__shfl_sync(0xffffffffu, a[e].x, k + 16 * hf),
                                      __shfl_sync(0xffffffffu, a[e].y, k + 16 * hf)), pinv);
                const bool colk = (hf == hk) && (e == ek);
                if (r == k) a[e] = colk ? pinv : pr;
                else if (colk) a[e] = zneg(zmul(f, pinv));
                else zfms(a[e], f, pr);
            }
        }
        // undo the column exchanges: X = X_pre P, column c of X is column sig(c) of X_pre;
        // piv[A + c'] receives the destination column of pre-column c'
        __syncwarp();
        if (lane == 0) {
            int sg[A];
            for (int c = 0; c < A; ++c) sg[c] = c;
            for (int k = A - 1; k >= 0; --k) {
                const int p = piv[k];
                const int t = sg[k];
                sg[k] = sg[p];
                sg[p] = t;
            }
            for (int c = 0; c < A; ++c) piv[A + sg[c]] = c;
        }
        __syncwarp();
#pragma unroll
        for (int e = 0; e < 8; ++e) sm[r + piv[A + hf * 8 + e] * A] = a[e];
        __syncwarp();
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            prev[e] = sm[r + (hf * 8 + e) * A];
            Sl[(size_t)j * AA + r + (hf * 8 + e) * A] = prev[e];
        }
        __syncwarp();
    }
    if (!ok && lane == 0) atomicOr(status, 1);

    // ---- S^T Z = C^T, one right-hand side per lane at a time ---------------------------------------
    for (int c = lane; c - lane < nb; c += 32) {
        const bool live = c < nb;
        int ax = 0, q1 = -1, q2 = -1;
        if (live) leaf_bpoint2(A, b, c, ax, q1, q2);
        const double hr = ax == 0 ? L.hx : L.hy;
        const double c1 = -3.0 / hr, c2 = (1.0 / 3.0) / hr;
        // Y(c, nb+s) = f_c Q(c, s): the backward sweep stores its final values already scaled
        const z fc = zmul(zmk(0.0, 2.0 * g.kb), ax == 0 ? L.rdx : L.rdy);
        z v[A];
#pragma unroll
        for (int i = 0; i < A; ++i) v[i] = zmk(0.0, 0.0);
        // forward: v_j = Sig_j^-T (c_j - Up_{j-1} v_{j-1})
        for (int j = 0; j < b; ++j) {
            const int jj = j + 1;
            const z mup = jj > 1 ? block_up(L, b, jj - 1) : zmk(0.0, 0.0);
            __syncwarp();
#pragma unroll
            for (int e = 0; e < 8; ++e) sm[r + (hf * 8 + e) * A] = Sl[(size_t)j * AA + r + (hf * 8 + e) * A];
            __syncwarp();
            z rhs[A];
#pragma unroll
            for (int q = 0; q < A; ++q) {
                const int eq = j * A + q;
                rhs[q] = zmk((eq == q1 ? c1 : 0.0) + (eq == q2 ? c2 : 0.0), 0.0);
                if (jj > 1) zfms(rhs[q], mup, v[q]);
            }
#pragma unroll
            for (int i = 0; i < A; ++i) {
                z acc = zmk(0.0, 0.0);
#pragma unroll
                for (int q = 0; q < A; ++q) zfma(acc, sm[q + i * A], rhs[q]);
                v[i] = acc;
                if (live) Yl[c + (size_t)(nb + j * A + i) * nb] = acc;
            }
        }
        // backward: z_{j-1} = v_{j-1} - Sig_{j-1}^-T Lo_j z_j, z_{b-1} = v_{b-1}
        if (live) {
#pragma unroll
            for (int i = 0; i < A; ++i) Yl[c + (size_t)(nb + (b - 1) * A + i) * nb] = zmul(fc, v[i]);
        }
        for (int j = b - 1; j >= 1; --j) {
            const z lam = block_lo(L, b, j + 1);
            __syncwarp();
#pragma unroll
            for (int e = 0; e < 8; ++e) sm[r + (hf * 8 + e) * A] = Sl[(size_t)(j - 1) * AA + r + (hf * 8 + e) * A];
            __syncwarp();
            z lz[A];
#pragma unroll
            for (int q = 0; q < A; ++q) lz[q] = zmul(lam, v[q]);
#pragma unroll
            for (int i = 0; i < A; ++i) {
                z acc = live ? Yl[c + (size_t)(nb + (j - 1) * A + i) * nb] : zmk(0.0, 0.0);
#pragma unroll
                for (int q = 0; q < A; ++q) zfms(acc, sm[q + i * A], lz[q]);
                v[i] = acc;
                if (live) Yl[c + (size_t)(nb + (j - 1) * A + i) * nb] = zmul(fc, acc);
            }
        }
    }
    __syncwarp();
    // ---- Y(:, 0:nb) from the scaled Y(r, nb+s) = f_r Q(r, s) ----------------------------------------
    for (int e = lane; e < nb * nb; e += 32) {
        const int rr = e % nb, c = e / nb;
        int ax, p1, p2, axc, q1, q2;
        leaf_bpoint2(A, b, rr, ax, p1, p2);
        leaf_bpoint2(A, b, c, axc, q1, q2);
        const z rd = ax == 0 ? L.rdx : L.rdy;
        const z wd = axc == 0 ? zscale(L.wbx, L.rdx) : zscale(L.wby, L.rdy);
        z val = zneg(zmul(wd, Yl[rr + (size_t)(nb + q1) * nb]));
        if (c == rr) {
            const double hr2 = ax == 0 ? L.hx : L.hy;
            val = zadd(val, zmul(zmk((8.0 / 3.0) / hr2, -g.kb), rd));
        }
        Yl[e] = val;
    }
}

size_t leaf_block_factor_smem(const LeafGeom& g) {
    return (2 * (size_t)g.a * g.a + 2 * (size_t)g.a * g.nb + g.a) * sizeof(z) + (g.a + 1) * sizeof(int) + 16;
}

// ---------------------------------------------------------------------------------------------------
// Tensor-core leaf factor for 16 x b leaves with nb <= 64 boundary points: one warp per leaf, the
// block LU of leaf_warp_factor_kernel, and the two sweeps of S^T Z = C^T as FP64 tensor-core
// products (mma.sync m8n8k4 .f64, four real products per complex one) over chunks of 32
// right-hand sides: block step j is V_j = Sig_j^-T R_j with R_j (16 x 32) in shared memory.
// The forward step of block j runs as soon as the LU has Sig_j^-1 in the warp's shared memory,
// so the forward sweep never reloads it; the backward sweep reloads one block per step.
//   forward:  R_0 = C_0;  V_j = Sig_j^-T R_j;  R_{j+1} = C_{j+1} - Up_j V_j
//   backward: Z_{b-1} = V_{b-1};  Z_{j-1} = V_{j-1} - Sig_{j-1}^-T (Lo_j Z_j)
// C_j holds, per right-hand side c, c1 and c2 at the interior points next to boundary point c.
constexpr int LTC_CH = 2;        // chunks of 32 right-hand sides (nb <= 64)
constexpr int LTC_LDR = 18;      // padded leading dimension of the R buffers (bank spread)

// acc (2 x 4 tiles of 8x8, complex as re/im) += A B,  A(i,k) = As[k + 16 i],  B(k,c) = Bs[k + LTC_LDR c]
__device__ __forceinline__ void ltc_mma(const z* As, const z* Bs, double (&cre)[2][4][2], double (&cim)[2][4][2],
                                        int lane) {
    const int lr = lane >> 2, lc = lane & 3;
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
        double ar[2], ai[2], nai[2], br[4], bi[4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
            const z a = As[(4 * ks + lc) + 16 * (8 * mi + lr)];
            ar[mi] = a.x;
            ai[mi] = a.y;
            nai[mi] = -a.y;
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
            const z b = Bs[(4 * ks + lc) + LTC_LDR * (8 * ni + lr)];
            br[ni] = b.x;
            bi[ni] = b.y;
        }
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma884(cre[mi][ni][0], cre[mi][ni][1], ar[mi], br[ni]);
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma884(cim[mi][ni][0], cim[mi][ni][1], ar[mi], bi[ni]);
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma884(cre[mi][ni][0], cre[mi][ni][1], nai[mi], bi[ni]);
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma884(cim[mi][ni][0], cim[mi][ni][1], ai[mi], br[ni]);
    }
}

// R_j's sparse part: lane c (a right-hand side of chunk ch) adds c1, c2 where its two interior
// points fall in block j (interior index q = 16 j + row)
__device__ __forceinline__ void ltc_add_c(z* R, int ch, int j, int lane, int b, int nb, const LeafConst& L) {
    const int c = 32 * ch + lane;
    if (c >= nb) return;
    int ax, q1, q2;
    leaf_bpoint2(16, b, c, ax, q1, q2);
    const double h = ax == 0 ? L.hx : L.hy;
    const double c1 = -3.0 / h, c2 = (1.0 / 3.0) / h;
    const int q0 = 16 * j;
    if (q1 >= q0 && q1 < q0 + 16) R[(q1 - q0) + LTC_LDR * lane].x += c1;
    if (q2 >= q0 && q2 < q0 + 16) R[(q2 - q0) + LTC_LDR * lane].x += c2;
}

__global__ void __launch_bounds__(128) leaf_tc_factor_kernel(LeafGeom g, int nleaves, const double* __restrict__ hh,
                                                             const z* __restrict__ kv, z* __restrict__ sinv,
                                                             z* __restrict__ Y, int* status) {
    constexpr int A = 16, AA = 256;
    extern __shared__ z ltc_smem[];
    __shared__ int wpiv[4][2 * A];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int leaf = blockIdx.x * 4 + wib;
    if (leaf >= nleaves) return;
    z* sm = ltc_smem + (size_t)wib * (AA + LTC_CH * LTC_LDR * 32);
    z* R = sm + AA;                                  // LTC_CH buffers of LTC_LDR x 32
    int* piv = wpiv[wib];
    const int b = g.b, nb = g.nb, n = g.n, ab = A * b;
    const int nch = (nb + 31) / 32;
    const LeafConst L = leaf_const(hh, leaf, g.kb);
    const z* kl = kv + (size_t)leaf * ab;
    z* Sl = sinv + (size_t)leaf * b * AA;
    z* Yl = Y + (size_t)leaf * nb * n;
    const int r = lane & 15, hf = lane >> 4;
    const int lr = lane >> 2, lc = lane & 3;
    z a[8], prev[8];
    bool ok = true;

    // R_0 = C_0
    for (int ch = 0; ch < nch; ++ch) {
        z* Rc = R + ch * LTC_LDR * 32;
        for (int e = lane; e < LTC_LDR * 32; e += 32) Rc[e] = zmk(0.0, 0.0);
        __syncwarp();
        ltc_add_c(Rc, ch, 0, lane, b, nb, L);
    }
    __syncwarp();

    for (int j = 0; j < b; ++j) {
        // ---- block LU step: Sig_j^-1 (leaf_warp_factor_kernel's Gauss-Jordan) -----------------------
        const int jj = j + 1;
        const z lm = jj > 1 ? zmul(block_lo(L, b, jj), block_up(L, b, jj - 1)) : zmk(0.0, 0.0);
        const z kr = kl[j * A + r];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            z v = block_d(L, A, b, jj, r, hf * 8 + e, kr);
            if (jj > 1) zfms(v, lm, prev[e]);
            a[e] = v;
        }
#pragma unroll
        for (int k = 0; k < A; ++k) {
            const int hk = k >> 3, ek = k & 7;
            double mag = (hf == hk && r >= k) ? zabs1(a[ek]) : -1.0;
            int idx = r;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double om = __shfl_xor_sync(0xffffffffu, mag, o);
                const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
                if (om > mag || (om == mag && oi < idx)) { mag = om; idx = oi; }
            }
            const int p = idx;
            if (lane == 0) piv[k] = p;
            if (p != k) {
                const int src = (r == k ? p : (r == p ? k : r)) + 16 * hf;
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const double x = __shfl_sync(0xffffffffu, a[e].x, src);
                    const double y = __shfl_sync(0xffffffffu, a[e].y, src);
                    a[e] = zmk(x, y);
                }
            }
            const z pv = zmk(__shfl_sync(0xffffffffu, a[ek].x, k + 16 * hk),
                             __shfl_sync(0xffffffffu, a[ek].y, k + 16 * hk));
            if (pv.x == 0.0 && pv.y == 0.0) ok = false;
            const z pinv = zrcp(pv);
            const z f = zmk(__shfl_sync(0xffffffffu, a[ek].x, r + 16 * hk),
                            __shfl_sync(0xffffffffu, a[ek].y, r + 16 * hk));
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const z pr = zmul(zmk(__shfl_sync(0xffffffffu, a[e].x, k + 16 * hf),
                                      __shfl_sync(0xffffffffu, a[e].y, k + 16 * hf)), pinv);
                const bool colk = (hf == hk) && (e == ek);
                if (r == k) a[e] = colk ? pinv : pr;
                else if (colk) a[e] = zneg(zmul(f, pinv));
                else zfms(a[e], f, pr);
            }
        }
        __syncwarp();
        if (lane == 0) {
            int sg[A];
            for (int c = 0; c < A; ++c) sg[c] = c;
            for (int k = A - 1; k >= 0; --k) {
                const int p = piv[k];
                const int t = sg[k];
                sg[k] = sg[p];
                sg[p] = t;
            }
            for (int c = 0; c < A; ++c) piv[A + sg[c]] = c;
        }
        __syncwarp();
#pragma unroll
        for (int e = 0; e < 8; ++e) sm[r + piv[A + hf * 8 + e] * A] = a[e];
        __syncwarp();
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            prev[e] = sm[r + (hf * 8 + e) * A];
            Sl[(size_t)j * AA + r + (hf * 8 + e) * A] = prev[e];
        }
        __syncwarp();
        // ---- forward step j for every chunk: V_j = Sig_j^-T R_j -----------------------------------
        const z mup = block_up(L, b, jj);            // Up_j, for R_{j+1}
        for (int ch = 0; ch < nch; ++ch) {
            z* Rc = R + ch * LTC_LDR * 32;
            double cre[2][4][2], cim[2][4][2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) cre[mi][ni][0] = cre[mi][ni][1] = cim[mi][ni][0] = cim[mi][ni][1] = 0.0;
            ltc_mma(sm, Rc, cre, cim, lane);
            __syncwarp();                              // every lane has read R_j
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int i = 8 * mi + lr, cl = 8 * ni + 2 * lc + h, c = 32 * ch + cl;
                        const z v = zmk(cre[mi][ni][h], cim[mi][ni][h]);
                        if (c < nb) Yl[c + (size_t)(nb + j * A + i) * nb] = v;
                        // next: R_{j+1} = C_{j+1} - Up_j V_j  (backward start: -Lo_b Z_{b-1})
                        Rc[i + LTC_LDR * cl] = zneg(zmul(jj < b ? mup : block_lo(L, b, b), v));
                    }
            __syncwarp();
            if (jj < b) ltc_add_c(Rc, ch, j + 1, lane, b, nb, L);
        }
        __syncwarp();
    }
    if (!ok && lane == 0) atomicOr(status, 1);

    // ---- backward sweep, Y(c, nb+s) = f_c Q(c, s) stored already scaled -------------------------------
    z fcl[4][2];                                      // f_c of this lane's columns, per chunk below
    for (int j = b - 1; j >= 0; --j) {
        // j >= 1: Z_{j-1} = V_{j-1} + Sig_{j-1}^-T R  with R = -Lo_j Z_j;  the final step (j = 0) only
        // rescales block... handled by storing Z_{b-1} first
        if (j == b - 1) {
            for (int ch = 0; ch < nch; ++ch) {
                // Z_{b-1} = V_{b-1}, scaled
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int i = 8 * mi + lr, c = 32 * ch + 8 * ni + 2 * lc + h;
                            if (c >= nb) continue;
                            int ax, q1, q2;
                            leaf_bpoint2(A, b, c, ax, q1, q2);
                            const z fc = zmul(zmk(0.0, 2.0 * g.kb), ax == 0 ? L.rdx : L.rdy);
                            z* yp = Yl + c + (size_t)(nb + j * A + i) * nb;
                            *yp = zmul(fc, *yp);
                        }
            }
        }
        if (j == 0) break;
#pragma unroll
        for (int e = 0; e < 8; ++e) sm[r + (hf * 8 + e) * A] = Sl[(size_t)(j - 1) * AA + r + (hf * 8 + e) * A];
        __syncwarp();
        const z lamn = j >= 2 ? block_lo(L, b, j) : zmk(0.0, 0.0);   // Lo_{j-1}, for the next step
        for (int ch = 0; ch < nch; ++ch) {
            z* Rc = R + ch * LTC_LDR * 32;
            double cre[2][4][2], cim[2][4][2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int i = 8 * mi + lr, c = 32 * ch + 8 * ni + 2 * lc + h;
                        const z v = c < nb ? Yl[c + (size_t)(nb + (j - 1) * A + i) * nb] : zmk(0.0, 0.0);
                        cre[mi][ni][h] = v.x;
                        cim[mi][ni][h] = v.y;
                        int ax, q1, q2;
                        leaf_bpoint2(A, b, c < nb ? c : 0, ax, q1, q2);
                        fcl[ni][h] = zmul(zmk(0.0, 2.0 * g.kb), ax == 0 ? L.rdx : L.rdy);
                    }
            ltc_mma(sm, Rc, cre, cim, lane);
            __syncwarp();
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int i = 8 * mi + lr, cl = 8 * ni + 2 * lc + h, c = 32 * ch + cl;
                        const z zv = zmk(cre[mi][ni][h], cim[mi][ni][h]);
                        if (c < nb) Yl[c + (size_t)(nb + (j - 1) * A + i) * nb] = zmul(fcl[ni][h], zv);
                        Rc[i + LTC_LDR * cl] = zneg(zmul(lamn, zv));
                    }
            __syncwarp();
        }
    }
    __syncwarp();
    // ---- Y(:, 0:nb) from the scaled Y(r, nb+s) = f_r Q(r, s) ----------------------------------------
    for (int e = lane; e < nb * nb; e += 32) {
        const int rr = e % nb, c = e / nb;
        int ax, p1, p2, axc, q1, q2;
        leaf_bpoint2(A, b, rr, ax, p1, p2);
        leaf_bpoint2(A, b, c, axc, q1, q2);
        const z rd = ax == 0 ? L.rdx : L.rdy;
        const z wd = axc == 0 ? zscale(L.wbx, L.rdx) : zscale(L.wby, L.rdy);
        z val = zneg(zmul(wd, Yl[rr + (size_t)(nb + q1) * nb]));
        if (c == rr) {
            const double hr2 = ax == 0 ? L.hx : L.hy;
            val = zadd(val, zmul(zmk((8.0 / 3.0) / hr2, -g.kb), rd));
        }
        Yl[e] = val;
    }
}

static bool leaf_tc_enabled() {
    const char* v = std::getenv("RB_LEAF_ENGINE");
    return !(v && v[0] == 'd');       // RB_LEAF_ENGINE=dfma: the DFMA warp kernel (comparisons)
}

cudaError_t leaf_block_factor(const LeafGeom& g, int nleaves, const double* h, const z* k, z* sinv, z* Y,
                              int* status, cudaStream_t s) {
    if (g.a == 16 && g.nb <= 32 * LTC_CH && leaf_tc_enabled()) {     // one warp per leaf, tensor cores
        const size_t sh = 4 * (256 + (size_t)LTC_CH * LTC_LDR * 32) * sizeof(z);
        static DeviceAttrCache attr;
        {
            cudaError_t e = ensure_smem_attr(leaf_tc_factor_kernel, sh, attr);
            if (e != cudaSuccess) return e;
        }
        leaf_tc_factor_kernel<<<(nleaves + 3) / 4, 128, sh, s>>>(g, nleaves, h, k, sinv, Y, status);
        note_launch();
        return cudaGetLastError();
    }
    if (g.a == 16) {                        // one warp per leaf
        leaf_warp_factor_kernel<<<(nleaves + 3) / 4, 128, 0, s>>>(g, nleaves, h, k, sinv, Y, status);
        note_launch();
        return cudaGetLastError();
    }
    const size_t sh = leaf_block_factor_smem(g);
    if (sh > 48 * 1024) {
        static DeviceAttrCache attr;
        cudaError_t e = ensure_smem_attr(leaf_block_factor_kernel, sh, attr);
        if (e != cudaSuccess) return e;
    }
    leaf_block_factor_kernel<<<nleaves, 256, sh, s>>>(g, h, k, sinv, Y, status);
    note_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------------
// Leaf solve: u = A^-1 [g; f] for every leaf and right-hand side into sol [rhs][leaf][n].
// RHS are processed in chunks of KC columns; shared memory: sig (a^2), w0, w1 (a x KC each).
constexpr int LEAF_KC = 32;

// leaf solve engine: the half-warp kernel for 16-point leaves (default) or the block kernel
// (RB_LEAF_SOLVE=block, read once; a comparison knob)
static bool leaf_solve_engine_hw() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("RB_LEAF_SOLVE");
        v = (e && std::strcmp(e, "block") == 0) ? 0 : 1;
    }
    return v == 1;
}

__global__ void __launch_bounds__(256) leaf_block_solve_kernel(LeafGeom g, int nleaves, int nrhs,
                                                               const double* __restrict__ hh,
                                                               const z* __restrict__ f, const z* __restrict__ gb,
                                                               const z* __restrict__ sinv, z* __restrict__ sol) {
    extern __shared__ z sm[];
    const int leaf = blockIdx.x;
    const int a = g.a, b = g.b, nb = g.nb, n = g.n, ab = a * b, aa = a * a;
    const int tid = threadIdx.x, nt = blockDim.x;
    z* sig = sm;
    z* w0 = sig + aa;
    z* w1 = w0 + (size_t)a * LEAF_KC;
    const LeafConst L = leaf_const(hh, leaf, g.kb);
    const z* Sl = sinv + (size_t)leaf * b * aa;
    const z wdx = zscale(L.wbx, L.rdx), wdy = zscale(L.wby, L.rdy);
    for (int r0 = 0; r0 < nrhs; r0 += LEAF_KC) {
        const int kc = min(LEAF_KC, nrhs - r0);
        z* wp = w0;
        z* wc = w1;
        // forward: w_j = Sig_j^-1 (t_j - Lo_j w_{j-1}),  t = f - A_ib A_bb^-1 g
        for (int j = 0; j < b; ++j) {
            const int jj = j + 1;
            for (int e = tid; e < aa; e += nt) sig[e] = Sl[(size_t)j * aa + e];
            const z lam = jj > 1 ? block_lo(L, b, jj) : zmk(0.0, 0.0);
            __syncthreads();
            // right-hand side of block j into wc (t_j - Lo_j w_{j-1})
            for (int e = tid; e < a * kc; e += nt) {
                const int q = e % a, rc = e / a, rh = r0 + rc;
                const int i = q + 1;
                const z* gl = gb + ((size_t)leaf * nrhs + rh) * nb;
                z t = f ? f[((size_t)rh * nleaves + leaf) * ab + j * a + q] : zmk(0.0, 0.0);
                if (i == 1) zfms(t, wdx, gl[j]);
                if (i == a) zfms(t, wdx, gl[b + j]);
                if (jj == 1) zfms(t, wdy, gl[2 * b + q]);
                if (jj == b) zfms(t, wdy, gl[2 * b + a + q]);
                if (jj > 1) zfms(t, lam, wp[q + rc * a]);
                wc[e] = t;
            }
            __syncthreads();
            for (int e = tid; e < a * kc; e += nt) {
                const int i = e % a, rc = e / a;
                z acc = zmk(0.0, 0.0);
                for (int q = 0; q < a; ++q) zfma(acc, sig[i + q * a], wc[q + rc * a]);
                sol[((size_t)(r0 + rc) * nleaves + leaf) * n + nb + j * a + i] = acc;
                wp[e] = acc;    // w_j becomes the previous block for j+1
            }
            __syncthreads();
        }
        // backward: x_{b-1} = w_{b-1} (in wp); x_j = w_j - Sig_j^-1 Up_j x_{j+1}
        for (int j = b - 2; j >= 0; --j) {
            const int jj = j + 1;
            const z mu = block_up(L, b, jj);
            for (int e = tid; e < aa; e += nt) sig[e] = Sl[(size_t)j * aa + e];
            __syncthreads();
            for (int e = tid; e < a * kc; e += nt) {
                const int i = e % a, rc = e / a;
                z* up = sol + ((size_t)(r0 + rc) * nleaves + leaf) * n + nb + j * a;
                z acc = up[i];
                for (int q = 0; q < a; ++q) zfms(acc, sig[i + q * a], zmul(mu, wp[q + rc * a]));
                wc[e] = acc;
                up[i] = acc;
            }
            __syncthreads();
            z* t = wp; wp = wc; wc = t;
        }
        __syncthreads();
        // boundary values u_b = (g - c1 u(p1) - c2 u(p2)) / d
        for (int e = tid; e < nb * kc; e += nt) {
            const int r = e % nb, rc = e / nb, rh = r0 + rc;
            int ax, p1, p2;
            leaf_bpoint2(a, b, r, ax, p1, p2);
            const double h = ax == 0 ? L.hx : L.hy;
            z* u = sol + ((size_t)rh * nleaves + leaf) * n;
            z v = gb[((size_t)leaf * nrhs + rh) * nb + r];
            v = zsub(v, zadd(zscale(-3.0 / h, u[nb + p1]), zscale((1.0 / 3.0) / h, u[nb + p2])));
            u[r] = zmul(v, ax == 0 ? L.rdx : L.rdy);
        }
        __syncthreads();
    }
}

// The same solve for leaves 16 points wide (a == 16), one CTA of 8 warps per leaf and 32
// right-hand sides at a time.  Each half-warp owns a right-hand side column, lane i its row i,
// so a block step's recurrence stays in the lane's registers and its 16-term products exchange
// values through shared memory within the warp.  The next step's Sig_j^-1 block and its right-hand
// side block (f_j forward, the stored w_j backward) are fetched with cp.async while the current
// step runs: one block barrier per step, which also releases the buffer the next fetch
// overwrites.  Same operations in the same order as leaf_block_solve_kernel.
constexpr int LHW_KC = 32;
__global__ void __launch_bounds__(256, 3) leaf_hw_solve_kernel(LeafGeom g, int nleaves, int nrhs,
                                                            const double* __restrict__ hh,
                                                            const z* __restrict__ f, const z* __restrict__ gb,
                                                            const z* __restrict__ sinv, z* __restrict__ sol) {
    constexpr int A = 16, AA = A * A, KC = LHW_KC, CPH = KC / 16;   // columns per half-warp
    extern __shared__ z sm[];
    const int leaf = blockIdx.x;
    const int b = g.b, nb = g.nb, n = g.n, ab = A * b;
    z* sig = sm;                       // [2][AA]: Sig_j^-1 of the current and the next step
    z* blk = sig + 2 * AA;             // [2][A*KC]: the steps' right-hand side blocks
    z* gsm = blk + 2 * A * KC;         // [KC][nb]: boundary data of the chunk
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int i = lane & 15, half = lane >> 4;
    const LeafConst L = leaf_const(hh, leaf, g.kb);
    const z* Sl = sinv + (size_t)leaf * b * AA;
    const z wdx = zscale(L.wbx, L.rdx), wdy = zscale(L.wby, L.rdy);
    const int nsteps = 2 * b - 1;      // forward blocks 0..b-1, then backward blocks b-2..0
    for (int r0 = 0; r0 < nrhs; r0 += KC) {
        const int kc = min(KC, nrhs - r0);
        auto issue = [&](int st) {
            const int j = st < b ? st : 2 * b - 2 - st;
            z* sd = sig + (st & 1) * AA;
            for (int e = tid; e < AA; e += 256) cp_async16(sd + e, Sl + (size_t)j * AA + e, 16);
            z* bd = blk + (st & 1) * A * KC;
            for (int e = tid; e < A * KC; e += 256) {
                const int q = e % A, rc = e / A, rh = r0 + rc;
                const z* src = nullptr;
                if (rc < kc) {
                    if (st >= b) src = sol + ((size_t)rh * nleaves + leaf) * n + nb + j * A + q;
                    else if (f) src = f + ((size_t)rh * nleaves + leaf) * ab + j * A + q;
                }
                cp_async16(bd + e, src ? src : Sl, src ? 16 : 0);
            }
        };
        for (int e = tid; e < nb * KC; e += 256) {
            const int r = e % nb, rc = e / nb;
            const bool ok = rc < kc;
            cp_async16(gsm + e, ok ? gb + ((size_t)leaf * nrhs + r0 + rc) * nb + r : gb, ok ? 16 : 0);
        }
        issue(0);
        cp_async_commit();
        z w[CPH];                      // this lane's entry of the running block vector per column
#pragma unroll
        for (int c = 0; c < CPH; ++c) w[c] = zmk(0.0, 0.0);
        for (int st = 0; st < nsteps; ++st) {
            cp_async_wait<0>();
            __syncthreads();           // step st's blocks landed; every thread is past step st-1
            if (st + 1 < nsteps) issue(st + 1);
            cp_async_commit();
            const z* S = sig + (st & 1) * AA;
            z* B = blk + (st & 1) * A * KC;
            if (st < b) {
                // forward: w_j = Sig_j^-1 (t_j - Lo_j w_{j-1}),  t = f - A_ib A_bb^-1 g
                const int j = st, jj = j + 1;
                const z lam = jj > 1 ? block_lo(L, b, jj) : zmk(0.0, 0.0);
#pragma unroll
                for (int c = 0; c < CPH; ++c) {
                    const int rc = warp * (2 * CPH) + half + 2 * c;
                    const z* gl = gsm + rc * nb;
                    z t = B[i + rc * A];
                    if (i == 0) zfms(t, wdx, gl[j]);
                    if (i == A - 1) zfms(t, wdx, gl[b + j]);
                    if (jj == 1) zfms(t, wdy, gl[2 * b + i]);
                    if (jj == b) zfms(t, wdy, gl[2 * b + A + i]);
                    if (jj > 1) zfms(t, lam, w[c]);
                    B[i + rc * A] = t;
                }
                __syncwarp();
                z acc[CPH];
#pragma unroll
                for (int c = 0; c < CPH; ++c) acc[c] = zmk(0.0, 0.0);
#pragma unroll
                for (int q = 0; q < A; ++q) {
                    const z sq = S[i + q * A];
#pragma unroll
                    for (int c = 0; c < CPH; ++c) zfma(acc[c], sq, B[q + (warp * (2 * CPH) + half + 2 * c) * A]);
                }
#pragma unroll
                for (int c = 0; c < CPH; ++c) {
                    const int rc = warp * (2 * CPH) + half + 2 * c;
                    w[c] = acc[c];
                    if (rc < kc) sol[((size_t)(r0 + rc) * nleaves + leaf) * n + nb + j * A + i] = acc[c];
                }
            } else {
                // backward: x_{b-1} = w_{b-1}; x_j = w_j - Sig_j^-1 Up_j x_{j+1}
                const int j = 2 * b - 2 - st;
                const z mu = block_up(L, b, j + 1);
                z wj[CPH];
#pragma unroll
                for (int c = 0; c < CPH; ++c) {
                    const int rc = warp * (2 * CPH) + half + 2 * c;
                    wj[c] = B[i + rc * A];
                    B[i + rc * A] = w[c];          // x_{j+1}, read by the other lanes of the half
                }
                __syncwarp();
#pragma unroll
                for (int q = 0; q < A; ++q) {
                    const z sq = S[i + q * A];
#pragma unroll
                    for (int c = 0; c < CPH; ++c)
                        zfms(wj[c], sq, zmul(mu, B[q + (warp * (2 * CPH) + half + 2 * c) * A]));
                }
#pragma unroll
                for (int c = 0; c < CPH; ++c) {
                    const int rc = warp * (2 * CPH) + half + 2 * c;
                    w[c] = wj[c];
                    if (rc < kc) sol[((size_t)(r0 + rc) * nleaves + leaf) * n + nb + j * A + i] = wj[c];
                }
            }
        }
        cp_async_wait<0>();
        __syncthreads();               // every interior value of the chunk is stored
        // boundary values u_b = (g - c1 u(p1) - c2 u(p2)) / d
        for (int e = tid; e < nb * kc; e += 256) {
            const int r = e % nb, rc = e / nb, rh = r0 + rc;
            int ax, p1, p2;
            leaf_bpoint2(A, b, r, ax, p1, p2);
            const double h = ax == 0 ? L.hx : L.hy;
            z* u = sol + ((size_t)rh * nleaves + leaf) * n;
            z v = gsm[rc * nb + r];
            v = zsub(v, zadd(zscale(-3.0 / h, u[nb + p1]), zscale((1.0 / 3.0) / h, u[nb + p2])));
            u[r] = zmul(v, ax == 0 ? L.rdx : L.rdy);
        }
        __syncthreads();               // the buffers are refilled for the next chunk
    }
}

cudaError_t leaf_block_solve(const LeafGeom& g, int nleaves, int nrhs, const double* h, const z* f, const z* gb,
                             const z* sinv, z* sol, cudaStream_t s) {
    if (g.a == 16 && leaf_solve_engine_hw()) {
        const size_t sh = ((size_t)2 * 256 + 2 * 16 * LHW_KC + (size_t)g.nb * LHW_KC) * sizeof(z);
        static DeviceAttrCache attr;
        {
            cudaError_t e = ensure_smem_attr(leaf_hw_solve_kernel, sh, attr);
            if (e != cudaSuccess) return e;
        }
        leaf_hw_solve_kernel<<<nleaves, 256, sh, s>>>(g, nleaves, nrhs, h, f, gb, sinv, sol);
        note_launch();
        return cudaGetLastError();
    }
    const size_t sh = ((size_t)g.a * g.a + 2 * (size_t)g.a * LEAF_KC) * sizeof(z);
    if (sh > 48 * 1024) {
        static DeviceAttrCache attr;
        cudaError_t e = ensure_smem_attr(leaf_block_solve_kernel, sh, attr);
        if (e != cudaSuccess) return e;
    }
    leaf_block_solve_kernel<<<nleaves, 256, sh, s>>>(g, nleaves, nrhs, h, f, gb, sinv, sol);
    note_launch();
    return cudaGetLastError();
}

}  // namespace rb
