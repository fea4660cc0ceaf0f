// rb_refine.cu -- FP64 residual of the global finite-difference system and the other kernels of
// the mixed-precision solve's iterative refinement.
//
// The HPS tree eliminates one global FD system whose unknowns are every leaf's u vector (its
// cornerless grid, lin2fgrid order).  Its rows, per leaf:
//   interior point e     (Delta_h u + k u)(e) = f(e)           FD_matrix_row, fd_module.f90:140-181
//   boundary point on the domain boundary      g_in(u) = g      fd_module.f90:187-216
//   boundary point on an interface             h_out(u) - zeta g_in(u) - nu g_in(u')(p') = 0
// with g_in = i kb u_b + D_n u and h_out = -i kb u_b + D_n u, D_n u = (8/3 u_b - 3 u_1 + 1/3 u_2)/h
// (RTR_update's sigma = -i kb, tau = 1, robin_tree_module.f90:683-713), and u' the neighbouring
// leaf's u at the same physical point (the transmission conditions the merge solves,
// robin_tree_module.f90:425-467).
//
// Refinement keeps the residual in place: with d the latest correction (or the first solution)
// and r the right-hand side it solved for, r <- r - A d is the residual of the accumulated
// solution.  Interior rows live in the solve's source array f, domain-boundary rows in the root's
// boundary data g, interface rows in their own array ri ([rhs][leaf][nb]); the correction sweep
// then adds -ri to the outgoing data h of each interface point at the level whose merge solves
// for it (iface_inject), because the interface equation of a merge reads
// (zeta - T_ii) g_i + nu g_i' = h_particular - r.
#include <cstdint>

#include "rb_kernels.h"

namespace rb {

namespace {

// position in a leaf's u vector of grid point (i, j): fgrid2lin (fd_module.f90:717-800)
__device__ __forceinline__ int leaf_lin(int i, int j, int a, int b) {
    const int nb = 2 * (a + b);
    if (i == 0) return j - 1;
    if (i == a + 1) return b + j - 1;
    if (j == 0) return 2 * b + i - 1;
    if (j == b + 1) return 2 * b + a + i - 1;
    return nb + (j - 1) * a + (i - 1);
}

// boundary row r: its grid point, the first two interior points along the inward normal, axis
__device__ __forceinline__ void leaf_bnd(int r, int a, int b, int& e1, int& e2, int& axis) {
    int i, j, si, sj;
    if (r < b) { i = 0; j = r + 1; si = 1; sj = 0; axis = 0; }
    else if (r < 2 * b) { i = a + 1; j = r - b + 1; si = -1; sj = 0; axis = 0; }
    else if (r < 2 * b + a) { i = r - 2 * b + 1; j = 0; si = 0; sj = 1; axis = 1; }
    else { i = r - 2 * b - a + 1; j = b + 1; si = 0; sj = -1; axis = 1; }
    e1 = leaf_lin(i + si, j + sj, a, b);
    e2 = leaf_lin(i + 2 * si, j + 2 * sj, a, b);
}

__device__ __forceinline__ z dn_u(const z* u, int r, int e1, int e2, double hn) {
    // (8/3 u_b - 3 u_1 + 1/3 u_2) / h, in the order fd_module.f90:207-215 adds the terms
    z v = zscale((8.0 / 3.0) / hn, u[r]);
    v = zadd(v, zscale(-3.0 / hn, u[e1]));
    v = zadd(v, zscale((1.0 / 3.0) / hn, u[e2]));
    return v;
}

__device__ __forceinline__ void atomic_max_nonneg(double* p, double v) {
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long*>(p), __double_as_longlong(v));
}

}  // namespace

// One CTA per RES_LEAVES consecutive leaves of one right-hand side (blockIdx.y).  d: the vector
// whose residual is taken ([rhs][leaf][n]); f: interior rows ([rhs][leaf][ab]), groot:
// domain-boundary rows ([rhs][root_nb]), ri: interface rows ([rhs][leaf][nb]), all updated in
// place (ri read as zero when first).  bclass[leaf*nb + r]: >= 0 the root boundary position of a
// domain-boundary point, < 0 -1 - (leaf'*nb + r') of the neighbour's row for the same point.
// rnorm[rhs]: max |r| over every row, accumulated with one atomic per CTA (one per warp and leaf
// serialised half a million atomics on the L2 slices holding rnorm).
constexpr int RES_LEAVES = 16;
constexpr int RES_THREADS = 128;
__global__ void __launch_bounds__(RES_THREADS) fd_residual_kernel(RefineGeom g, const z* __restrict__ d, z* f,
                                                                 z* groot, z* ri, const z* __restrict__ kv,
                                                                 const double* __restrict__ hh,
                                                                 const int* __restrict__ bclass, int first,
                                                                 double* rnorm) {
    extern __shared__ z ush[];
    __shared__ double wmax[RES_THREADS / 32];
    const int rhs = blockIdx.y;
    const int a = g.a, b = g.b, nb = 2 * (a + b), ab = a * b, n = nb + ab;
    const z ikb = zmk(0.0, g.kb), mikb = zmk(0.0, -g.kb);
    double mx = 0.0;
    const int l0 = blockIdx.x * RES_LEAVES;
    const int l1 = min(g.nleaves, l0 + RES_LEAVES);
    for (int leaf = l0; leaf < l1; ++leaf) {
        const z* u = d + ((long long)rhs * g.nleaves + leaf) * n;
        __syncthreads();                       // the previous leaf's reads of ush are done
        for (int e = threadIdx.x; e < n; e += blockDim.x) ush[e] = u[e];
        __syncthreads();
        const double hx = hh[2 * leaf], hy = hh[2 * leaf + 1];
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            if (e >= nb) {
                const int q = e - nb;
                const int gi = q % a + 1, gj = q / a + 1;
                z acc = zmul(kv[(long long)leaf * ab + q], ush[e]);
                // x then y, each the [w0, w1, w2] stencil of FD_matrix_row (fd_module.f90:150-181)
                for (int dim = 0; dim < 2; ++dim) {
                    const int gg = dim == 0 ? gi : gj, len = dim == 0 ? a : b;
                    double w0 = 1.0, w1 = -2.0, w2 = 1.0;
                    if (gg == 1) { w0 = 8.0 / 3.0; w1 = -4.0; w2 = 4.0 / 3.0; }
                    else if (gg == len) { w0 = 4.0 / 3.0; w1 = -4.0; w2 = 8.0 / 3.0; }
                    const double h2 = dim == 0 ? hx * hx : hy * hy;
                    const int eu = dim == 0 ? leaf_lin(gi + 1, gj, a, b) : leaf_lin(gi, gj + 1, a, b);
                    const int ed = dim == 0 ? leaf_lin(gi - 1, gj, a, b) : leaf_lin(gi, gj - 1, a, b);
                    acc = zadd(acc, zscale(w1 / h2, ush[e]));
                    acc = zadd(acc, zscale(w2 / h2, ush[eu]));
                    acc = zadd(acc, zscale(w0 / h2, ush[ed]));
                }
                z* fp = f + ((long long)rhs * g.nleaves + leaf) * ab + q;
                const z r = zsub(*fp, acc);
                *fp = r;
                mx = fmax(mx, fabs(r.x) + fabs(r.y));
            } else {
                int e1, e2, axis;
                leaf_bnd(e, a, b, e1, e2, axis);
                const double hn = axis == 0 ? hx : hy;
                const z dn = dn_u(ush, e, e1, e2, hn);
                const z gin = zadd(zmul(ikb, ush[e]), dn);
                const int cls = bclass[(long long)leaf * nb + e];
                z r;
                if (cls >= 0) {
                    z* gp = groot + (long long)rhs * g.root_nb + cls;
                    r = zsub(*gp, gin);
                    *gp = r;
                } else {
                    const int other = -1 - cls;
                    const int lj = other / nb, rj = other % nb;
                    const z* un = d + ((long long)rhs * g.nleaves + lj) * n;
                    int f1, f2, ax2;
                    leaf_bnd(rj, a, b, f1, f2, ax2);
                    const double hn2 = ax2 == 0 ? hh[2 * lj] : hh[2 * lj + 1];
                    z dn2 = zscale((8.0 / 3.0) / hn2, un[rj]);
                    dn2 = zadd(dn2, zscale(-3.0 / hn2, un[f1]));
                    dn2 = zadd(dn2, zscale((1.0 / 3.0) / hn2, un[f2]));
                    const z gin2 = zadd(zmul(ikb, un[rj]), dn2);
                    const z hout = zadd(zmul(mikb, ush[e]), dn);
                    // transmission row: h_out - zeta g_in - nu g_in' = 0
                    const z row = zsub(zsub(hout, zmul(g.zeta, gin)), zmul(g.nu, gin2));
                    z* rp = ri + ((long long)rhs * g.nleaves + leaf) * nb + e;
                    r = first ? zneg(row) : zsub(*rp, row);
                    *rp = r;
                }
                mx = fmax(mx, fabs(r.x) + fabs(r.y));
            }
        }
    }
    // max over the CTA, then over CTAs
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0 && rnorm) {
        for (int w = 1; w < RES_THREADS / 32; ++w) mx = fmax(mx, wmax[w]);
        atomic_max_nonneg(rnorm + rhs, mx);
    }
}

// hbuf (children of level l's nodes, [child][rhs column][nbc]) -= ri at the interface points:
// rows[(node*2 + k)*m + t] is the leaf boundary row (leaf*nb + r) of child k's interface point t.
__global__ void iface_inject_kernel(int nnodes, int m, int nbc, int o1, int o2, int nrhs, int leaf_rows,
                                    const int* __restrict__ rows, const z* __restrict__ ri, z* hbuf) {
    const long long tot = (long long)nnodes * 2 * m * nrhs;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const int t = (int)(e % m);
        long long q = e / m;
        const int k = (int)(q % 2);
        q /= 2;
        const int node = (int)(q % nnodes);
        const int r = (int)(q / nnodes);
        const int child = 2 * node + k;
        const int src = rows[((long long)node * 2 + k) * m + t];
        z* hp = hbuf + ((long long)child * nrhs + r) * nbc + (k == 0 ? o1 : o2) + t;
        *hp = zsub(*hp, ri[(long long)r * leaf_rows + src]);
    }
}

// x += dx over nrhs vectors of `per` elements; xnorm[r] = max |x|, dnorm[r] = max |dx| (|re|+|im|)
__global__ void refine_update_kernel(z* x, const z* __restrict__ dx, long long per, int nrhs, double* xnorm,
                                     double* dnorm) {
    const int r = blockIdx.y;
    double mx = 0.0, md = 0.0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < per; e += (long long)gridDim.x * blockDim.x) {
        const long long o = (long long)r * per + e;
        const z dv = dx[o];
        const z v = zadd(x[o], dv);
        x[o] = v;
        mx = fmax(mx, fabs(v.x) + fabs(v.y));
        md = fmax(md, fabs(dv.x) + fabs(dv.y));
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomic_max_nonneg(xnorm + r, mx);
        atomic_max_nonneg(dnorm + r, md);
    }
}

cudaError_t fd_residual(const RefineGeom& g, int nrhs, const z* d, z* f, z* groot, z* ri, const z* kv,
                        const double* hh, const int* bclass, bool first, double* rnorm, cudaStream_t s) {
    const int n = 2 * (g.a + g.b) + g.a * g.b;
    const size_t sh = (size_t)n * sizeof(z);
    if (sh > 48 * 1024) {
        static DeviceAttrCache attr;
        cudaError_t e = ensure_smem_attr(fd_residual_kernel, sh, attr);
        if (e != cudaSuccess) return e;
    }
    fd_residual_kernel<<<dim3((g.nleaves + RES_LEAVES - 1) / RES_LEAVES, nrhs), RES_THREADS, sh, s>>>(
        g, d, f, groot, ri, kv, hh, bclass, first ? 1 : 0, rnorm);
    note_launch();
    return cudaGetLastError();
}

cudaError_t iface_inject(int nnodes, int m, int nbc, int o1, int o2, int nrhs, int leaf_rows, const int* rows,
                         const z* ri, z* hbuf, cudaStream_t s) {
    const long long tot = (long long)nnodes * 2 * m * nrhs;
    const int blocks = (int)std::min<long long>((tot + 255) / 256, 148 * 8);
    iface_inject_kernel<<<blocks, 256, 0, s>>>(nnodes, m, nbc, o1, o2, nrhs, leaf_rows, rows, ri, hbuf);
    note_launch();
    return cudaGetLastError();
}

cudaError_t refine_update(z* x, const z* dx, long long per, int nrhs, double* xnorm, double* dnorm, cudaStream_t s) {
    const int bx = (int)std::min<long long>((per + 255) / 256, 4 * 148 / std::max(1, nrhs) + 1);
    refine_update_kernel<<<dim3(bx, nrhs), 256, 0, s>>>(x, dx, per, nrhs, xnorm, dnorm);
    note_launch();
    return cudaGetLastError();
}

}  // namespace rb
