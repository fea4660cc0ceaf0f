// rb_aux.cu -- leaf FD operator, merge and sweep helper kernels for sm_100a.
//
// Leaf algebra.  The reference's leaf matrix A (FD_matrix_row, fd_module.f90:104-224) has its
// rows/columns in lin2fgrid order: the nb = 2(a+b) cornerless boundary points first (faces
// x1 x2 y1 y2), then the a*b interior points x-fastest.  Every boundary row r reads only
// itself and two interior points along the inward normal:
//     A(r,r) = i*kb + (8/3)/h,  A(r,p1) = -3/h,  A(r,p2) = (1/3)/h        (fd_module.f90:207-215)
// so A_bb is diagonal and the boundary unknowns condense exactly.  With
// d_r = A(r,r), c1 = -3/h, c2 = 1/(3h) and w_c = (8/3)/h^2 (the interior row next to boundary
// point c couples to it with that weight, fd_module.f90:150-153):
//     S      = A_ii - A_ib A_bb^-1 A_bi                       (a*b x a*b, inverted by Gauss-Jordan)
//     A^-1   = [[ (I - A_bi A^-1_ib) / d ,  -A_bi S^-1 / d ],
//               [ -S^-1 A_ib / d          ,   S^-1          ]]
// The reference's leaf Robin-to-Robin map is R X with X = A^-1 [I; 0] and R the outgoing rows
// sigma*u + tau*(8/3 u - 3 u_p1 + 1/3 u_p2)/h, sigma = -i*kb, tau = 1
// (RTR_update, robin_tree_module.f90:683-713).  Row r of Y = R A^-1 is
//     Y(r,:) = (sigma'_r / d_r) e_r + (2 i kb / d_r) (c1 A^-1(p1,:) + c2 A^-1(p2,:)),
// sigma'_r = sigma + (8/3)/h, because sigma'_r - d_r = -2 i kb.  Y(:, 0:nb) is the leaf RtR,
// Y(:, nb:n) maps an interior source to the outgoing data of the particular solution
// (fd_leaf_solve + fd_outgoing_bc, fd_module.f90:390-513).
#include "rb_kernels.h"

namespace rb {

// boundary point r of an a x b leaf: normal axis and the first/second interior points along the
// inward normal, as 0-based interior indices ((j-1)*a + (i-1))
__device__ __forceinline__ void leaf_bpoint(int a, int b, int r, int& axis, int& p1, int& p2) {
    if (r < b) {                 // x1: (0, j)
        const int j = r;
        axis = 0; p1 = j * a; p2 = j * a + 1;
    } else if (r < 2 * b) {      // x2: (a+1, j)
        const int j = r - b;
        axis = 0; p1 = j * a + (a - 1); p2 = j * a + (a - 2);
    } else if (r < 2 * b + a) {  // y1: (i, 0)
        const int i = r - 2 * b;
        axis = 1; p1 = i; p2 = a + i;
    } else {                     // y2: (i, b+1)
        const int i = r - 2 * b - a;
        axis = 1; p1 = (b - 1) * a + i; p2 = (b - 2) * a + i;
    }
}

// 1D stencil weights of FD_matrix_row for grid index i in 1..a (fd_module.f90:150-156)
__device__ __forceinline__ void stencil(int i, int a, double& wm, double& w0, double& wp) {
    if (i == 1) { wm = 8.0 / 3.0; w0 = -4.0; wp = 4.0 / 3.0; }
    else if (i == a) { wm = 4.0 / 3.0; w0 = -4.0; wp = 8.0 / 3.0; }
    else { wm = 1.0; w0 = -2.0; wp = 1.0; }
}

__device__ __forceinline__ z bdiag(double h, double kb) {   // A(r,r) = i*kb + (8/3)/h
    return zmk((8.0 / 3.0) / h, kb);
}

// ---------------------------------------------------------------------------------------------------
__global__ void leaf_schur_kernel(LeafGeom g, const double* __restrict__ hh, const z* __restrict__ kv,
                                  z* __restrict__ S) {
    const int leaf = blockIdx.y;
    const int a = g.a, b = g.b, ab = a * b;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)ab * ab) return;
    const int e = (int)(idx % ab), c = (int)(idx / ab);
    const double hx = hh[2 * leaf], hy = hh[2 * leaf + 1];
    const double hx2 = hx * hx, hy2 = hy * hy;
    const int i = e % a + 1, j = e / a + 1;
    double wxm, wx0, wxp, wym, wy0, wyp;
    stencil(i, a, wxm, wx0, wxp);
    stencil(j, b, wym, wy0, wyp);
    const double wbx = (8.0 / 3.0) / hx2, wby = (8.0 / 3.0) / hy2;   // weight on a boundary neighbour
    const z rdx = zrcp(bdiag(hx, g.kb)), rdy = zrcp(bdiag(hy, g.kb));
    const double c1x = -3.0 / hx, c2x = (1.0 / 3.0) / hx, c1y = -3.0 / hy, c2y = (1.0 / 3.0) / hy;
    z v = zmk(0.0, 0.0);
    if (c == e) {
        const z k = kv[(long long)leaf * ab + e];
        v = zmk((k.x + wx0 / hx2) + wy0 / hy2, k.y);
        if (i == 1 || i == a) v = zsub(v, zscale(wbx * c1x, rdx));
        if (j == 1 || j == b) v = zsub(v, zscale(wby * c1y, rdy));
    } else if (i < a && c == e + 1) {
        v = zmk(wxp / hx2, 0.0);
        if (i == 1) v = zsub(v, zscale(wbx * c2x, rdx));
    } else if (i > 1 && c == e - 1) {
        v = zmk(wxm / hx2, 0.0);
        if (i == a) v = zsub(v, zscale(wbx * c2x, rdx));
    } else if (j < b && c == e + a) {
        v = zmk(wyp / hy2, 0.0);
        if (j == 1) v = zsub(v, zscale(wby * c2y, rdy));
    } else if (j > 1 && c == e - a) {
        v = zmk(wym / hy2, 0.0);
        if (j == b) v = zsub(v, zscale(wby * c2y, rdy));
    }
    S[(long long)leaf * ab * ab + idx] = v;
}

cudaError_t leaf_schur(const LeafGeom& g, int nleaves, const double* h, const z* k, z* S, cudaStream_t s) {
    const long long ab2 = (long long)g.a * g.b * g.a * g.b;
    dim3 grid((unsigned)((ab2 + 255) / 256), nleaves);
    leaf_schur_kernel<<<grid, 256, 0, s>>>(g, h, k, S);
    note_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------------
__global__ void leaf_outgoing_kernel(LeafGeom g, const double* __restrict__ hh, const z* __restrict__ Sinv,
                                     z* __restrict__ Y) {
    const int leaf = blockIdx.y;
    const int a = g.a, b = g.b, ab = a * b, nb = g.nb, n = g.n;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nb * n) return;
    const int r = (int)(idx % nb), col = (int)(idx / nb);
    const double hxy[2] = {hh[2 * leaf], hh[2 * leaf + 1]};
    const z* Si = Sinv + (long long)leaf * ab * ab;
    int ax, p1, p2;
    leaf_bpoint(a, b, r, ax, p1, p2);
    const double h = hxy[ax];
    const z rd = zrcp(bdiag(h, g.kb));
    const double c1 = -3.0 / h, c2 = (1.0 / 3.0) / h;
    const z fac = zmul(zmk(0.0, 2.0 * g.kb), rd);     // (d_r - sigma'_r) / d_r
    z v;
    if (col >= nb) {
        const int s = col - nb;
        const z q = zadd(zscale(c1, Si[p1 + (long long)s * ab]), zscale(c2, Si[p2 + (long long)s * ab]));
        v = zmul(fac, q);
    } else {
        int axc, p1c, p2c;
        leaf_bpoint(a, b, col, axc, p1c, p2c);
        const double hc = hxy[axc];
        const z wd = zscale((8.0 / 3.0) / (hc * hc), zrcp(bdiag(hc, g.kb)));   // w_c / d_c
        const z q = zadd(zscale(c1, Si[p1 + (long long)p1c * ab]), zscale(c2, Si[p2 + (long long)p1c * ab]));
        v = zneg(zmul(zmul(fac, wd), q));
        if (col == r) v = zadd(v, zmul(zmk((8.0 / 3.0) / h, -g.kb), rd));   // sigma'_r / d_r
    }
    Y[(long long)leaf * nb * n + idx] = v;
}

cudaError_t leaf_outgoing(const LeafGeom& g, int nleaves, const double* h, const z* Sinv, z* Y,
                          cudaStream_t s) {
    const long long tot = (long long)g.nb * g.n;
    dim3 grid((unsigned)((tot + 255) / 256), nleaves);
    leaf_outgoing_kernel<<<grid, 256, 0, s>>>(g, h, Sinv, Y);
    note_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------------
// t(e, r) = f(e) - sum over boundary neighbours c of e of (w_c / d_c) g(c)
__global__ void leaf_condense_rhs_kernel(LeafGeom g, int nleaves, int nrhs, const double* __restrict__ hh,
                                         const z* __restrict__ f, const z* __restrict__ gb, z* __restrict__ t) {
    const int leaf = blockIdx.y;
    const int a = g.a, b = g.b, ab = a * b, nb = g.nb;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)ab * nrhs) return;
    const int e = (int)(idx % ab), rh = (int)(idx / ab);
    const double hx = hh[2 * leaf], hy = hh[2 * leaf + 1];
    const int i = e % a + 1, j = e / a + 1;
    z v = f ? f[((long long)rh * nleaves + leaf) * ab + e] : zmk(0.0, 0.0);
    const z* gl = gb + ((long long)leaf * nrhs + rh) * nb;
    const z wdx = zscale((8.0 / 3.0) / (hx * hx), zrcp(bdiag(hx, g.kb)));
    const z wdy = zscale((8.0 / 3.0) / (hy * hy), zrcp(bdiag(hy, g.kb)));
    if (i == 1) zfms(v, wdx, gl[j - 1]);
    if (i == a) zfms(v, wdx, gl[b + j - 1]);
    if (j == 1) zfms(v, wdy, gl[2 * b + i - 1]);
    if (j == b) zfms(v, wdy, gl[2 * b + a + i - 1]);
    t[((long long)leaf * nrhs + rh) * ab + e] = v;
}

cudaError_t leaf_condense_rhs(const LeafGeom& g, int nleaves, int nrhs, const double* h, const z* f,
                              const z* gb, z* t, cudaStream_t s) {
    const long long tot = (long long)g.a * g.b * nrhs;
    dim3 grid((unsigned)((tot + 255) / 256), nleaves);
    leaf_condense_rhs_kernel<<<grid, 256, 0, s>>>(g, nleaves, nrhs, h, f, gb, t);
    note_launch();
    return cudaGetLastError();
}

// u_b(r) = (g(r) - c1 u(p1) - c2 u(p2)) / d_r, in place in the solution [rhs][leaf][n]
__global__ void leaf_boundary_values_kernel(LeafGeom g, int nleaves, int nrhs, const double* __restrict__ hh,
                                            const z* __restrict__ gb, z* __restrict__ sol) {
    const int leaf = blockIdx.y;
    const int a = g.a, b = g.b, nb = g.nb, n = g.n;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nb * nrhs) return;
    const int r = (int)(idx % nb), rh = (int)(idx / nb);
    int ax, p1, p2;
    leaf_bpoint(a, b, r, ax, p1, p2);
    const double h = hh[2 * leaf + ax];
    z* u = sol + ((long long)rh * nleaves + leaf) * n;
    z v = gb[((long long)leaf * nrhs + rh) * nb + r];
    v = zsub(v, zadd(zscale(-3.0 / h, u[nb + p1]), zscale((1.0 / 3.0) / h, u[nb + p2])));
    u[r] = zmul(v, zrcp(bdiag(h, g.kb)));
}

cudaError_t leaf_boundary_values(const LeafGeom& g, int nleaves, int nrhs, const double* h, const z* gb,
                                 z* sol, cudaStream_t s) {
    const long long tot = (long long)g.nb * nrhs;
    dim3 grid((unsigned)((tot + 255) / 256), nleaves);
    leaf_boundary_values_kernel<<<grid, 256, 0, s>>>(g, nleaves, nrhs, h, gb, sol);
    note_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------------
// D = zeta*I - T2_ii  (robin_tree_module.f90:440-446)
__global__ void merge_form_d_kernel(ChildStore c, int m, int o2, z zeta, z* __restrict__ dst) {
    const int node = blockIdx.y;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= m * m) return;
    const int r = idx % m, q = idx / m;
    const z* t2 = c.rtr + (long long)(2 * node + 1) * c.stride;
    z v = zneg(t2[(o2 + r) + (long long)(o2 + q) * c.ld]);
    if (r == q) v = zadd(v, zeta);
    dst[(long long)node * m * m + idx] = v;
}

// S = zeta*I - T1_ii - nu^2 inv(D)  (robin_tree_module.f90:457-464)
__global__ void merge_form_s_kernel(ChildStore c, int m, int o1, z zeta, z nu2, const z* __restrict__ dinv,
                                    z* __restrict__ dst) {
    const int node = blockIdx.y;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= m * m) return;
    const int r = idx % m, q = idx / m;
    const z* t1 = c.rtr + (long long)(2 * node) * c.stride;
    z v = zneg(t1[(o1 + r) + (long long)(o1 + q) * c.ld]);
    zfms(v, nu2, dinv[(long long)node * m * m + idx]);
    if (r == q) v = zadd(v, zeta);
    dst[(long long)node * m * m + idx] = v;
}

cudaError_t merge_form_d(ChildStore c, int nnodes, int m, int o2, z zeta, z* dst, cudaStream_t s) {
    dim3 grid((m * m + 255) / 256, nnodes);
    merge_form_d_kernel<<<grid, 256, 0, s>>>(c, m, o2, zeta, dst);
    note_launch();
    return cudaGetLastError();
}

cudaError_t merge_form_s(ChildStore c, int nnodes, int m, int o1, z zeta, z nu, const z* dinv, z* dst,
                         cudaStream_t s) {
    dim3 grid((m * m + 255) / 256, nnodes);
    merge_form_s_kernel<<<grid, 256, 0, s>>>(c, m, o1, zeta, zmul(nu, nu), dinv, dst);
    note_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------------
// backward sweep: children's non-interface g from the parent's g (robin_tree_module.f90:1045-1075)
__global__ void sweep_scatter_down_kernel(int nrhs, int nbp, int nbc, int m, int o1, int o2, int n1, int n2,
                                          const int* __restrict__ pmap1, const int* __restrict__ pmap2,
                                          const z* __restrict__ gpar, z* __restrict__ gchild) {
    const int node = blockIdx.y;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int per = n1 + n2;
    if (idx >= per * nrhs) return;
    const int t = idx % per, rh = idx / per;
    const z* gp = gpar + ((long long)node * nrhs + rh) * nbp;
    if (t < n1) {
        const int phys = t < o1 ? t : t + m;
        gchild[((long long)(2 * node) * nrhs + rh) * nbc + phys] = gp[pmap1[t]];
    } else {
        const int tt = t - n1;
        const int phys = tt < o2 ? tt : tt + m;
        gchild[((long long)(2 * node + 1) * nrhs + rh) * nbc + phys] = gp[pmap2[tt]];
    }
}

cudaError_t sweep_scatter_down(int nnodes, int nrhs, int nbp, int nbc, int m, int o1, int o2, int n1, int n2,
                               const int* pmap1, const int* pmap2, const z* gpar, z* gchild, cudaStream_t s) {
    const int tot = (n1 + n2) * nrhs;
    dim3 grid((tot + 255) / 256, nnodes);
    sweep_scatter_down_kernel<<<grid, 256, 0, s>>>(nrhs, nbp, nbc, m, o1, o2, n1, n2, pmap1, pmap2, gpar, gchild);
    note_launch();
    return cudaGetLastError();
}

// g_i += M^-1 (Tg): tmp per node = [tg1 | tg2 | y2 | y1], each m x nrhs (ld m)
__global__ void sweep_add_interface_kernel(int nrhs, int nbc, int m, int o1, int o2, const z* __restrict__ tmp,
                                           z* __restrict__ gchild) {
    const int node = blockIdx.y;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= m * nrhs) return;
    const int r = idx % m, rh = idx / m;
    const z* tb = tmp + (long long)node * 4 * m * nrhs;
    const z y2 = tb[2LL * m * nrhs + idx];
    const z y1 = tb[3LL * m * nrhs + idx];
    z* g1 = gchild + ((long long)(2 * node) * nrhs + rh) * nbc + o1 + r;
    z* g2 = gchild + ((long long)(2 * node + 1) * nrhs + rh) * nbc + o2 + r;
    *g1 = zadd(*g1, y1);
    *g2 = zadd(*g2, y2);
}

cudaError_t sweep_add_interface(int nnodes, int nrhs, int nbc, int m, int o1, int o2, const z* tmp, z* gchild,
                                cudaStream_t s) {
    dim3 grid((m * nrhs + 255) / 256, nnodes);
    sweep_add_interface_kernel<<<grid, 256, 0, s>>>(nrhs, nbc, m, o1, o2, tmp, gchild);
    note_launch();
    return cudaGetLastError();
}

}  // namespace rb
