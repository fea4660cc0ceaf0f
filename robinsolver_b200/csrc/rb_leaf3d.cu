// rb_leaf3d.cu -- the 3D (d = 3) finite-difference leaf: its dense matrix, the Robin-to-Robin rows
// of its inverse.  The inverse itself comes from the batched Gauss-Jordan kernels (rb_gj.cu) and
// the leaf solve u = A^-1 [g; f] from the batched GEMMs (rb_gemm.cu).
//
// Leaf layout (fd_module.f90:717-939 with d = 3): a x b x c interior points and, without edges or
// corners, the six faces x1 x2 (b c points each), y1 y2 (a c), z1 z2 (a b), each in its own 2D
// lexicographic order (first tangential index fastest), then the interior x fastest, then y, z.
// Rows (FD_matrix_row, fd_module.f90:104-224): on a face point, i kb u + (8/3 u0 - 3 u1 + 1/3 u2)/h
// along the inward normal; inside, k u plus the 1D stencil in x, y and z ([1, -2, 1] / h^2, or
// [8/3, -4, 4/3] / h^2 next to a face), added in that order.  The leaf's Robin-to-Robin rows
// (RTR_update, robin_tree_module.f90:667-718) replace each face row of A^-1 by
// -i kb X(r) + (8/3 X(r) - 3 X(r+s) + 1/3 X(r+2s)) / h.
#include "rb_kernels.h"

namespace rb {

namespace {

// fgrid2lin (fd_module.f90:717-800) for d = 3, 0-based; -1 for an edge or corner point
__device__ __forceinline__ int lin3(int i, int j, int k, int a, int b, int c) {
    const int bc = b * c, ac = a * c, ab = a * b;
    const int onx = (i == 0) + (i == a + 1), ony = (j == 0) + (j == b + 1), onz = (k == 0) + (k == c + 1);
    if (onx + ony + onz > 1) return -1;
    if (i == 0) return (k - 1) * b + (j - 1);
    if (i == a + 1) return bc + (k - 1) * b + (j - 1);
    if (j == 0) return 2 * bc + (k - 1) * a + (i - 1);
    if (j == b + 1) return 2 * bc + ac + (k - 1) * a + (i - 1);
    if (k == 0) return 2 * bc + 2 * ac + (j - 1) * a + (i - 1);
    if (k == c + 1) return 2 * bc + 2 * ac + ab + (j - 1) * a + (i - 1);
    return 2 * (bc + ac + ab) + ((k - 1) * b + (j - 1)) * a + (i - 1);
}

// lin2fgrid for d = 3, 0-based linear index -> (i, j, k)
__device__ __forceinline__ void grid3(int e, int a, int b, int c, int& i, int& j, int& k) {
    const int bc = b * c, ac = a * c, ab = a * b, nb = 2 * (bc + ac + ab);
    if (e < 2 * bc) {
        const int q = e % bc;
        i = e < bc ? 0 : a + 1; j = q % b + 1; k = q / b + 1;
    } else if (e < 2 * bc + 2 * ac) {
        const int q = (e - 2 * bc) % ac;
        j = e - 2 * bc < ac ? 0 : b + 1; i = q % a + 1; k = q / a + 1;
    } else if (e < nb) {
        const int q = (e - 2 * bc - 2 * ac) % ab;
        k = e - 2 * bc - 2 * ac < ab ? 0 : c + 1; i = q % a + 1; j = q / a + 1;
    } else {
        const int q = e - nb;
        i = q % a + 1; j = (q / a) % b + 1; k = q / (a * b) + 1;
    }
}

// face point r: the first and second points along the inward normal, and the normal axis
__device__ __forceinline__ void bnd3(int r, int a, int b, int c, int& p1, int& p2, int& axis) {
    int i, j, k;
    grid3(r, a, b, c, i, j, k);
    int si = 0, sj = 0, sk = 0;
    if (i == 0) { si = 1; axis = 0; }
    else if (i == a + 1) { si = -1; axis = 0; }
    else if (j == 0) { sj = 1; axis = 1; }
    else if (j == b + 1) { sj = -1; axis = 1; }
    else if (k == 0) { sk = 1; axis = 2; }
    else { sk = -1; axis = 2; }
    p1 = lin3(i + si, j + sj, k + sk, a, b, c);
    p2 = lin3(i + 2 * si, j + 2 * sj, k + 2 * sk, a, b, c);
}

}  // namespace

// One CTA per leaf: the dense n x n matrix (column-major) from the leaf's spacings hh (3 per leaf)
// and its potential samples kv (a b c per leaf, x fastest).
__global__ void __launch_bounds__(256) leaf3_assemble_kernel(Leaf3Geom g, const double* __restrict__ hh,
                                                             const z* __restrict__ kv, z* A) {
    const int leaf = blockIdx.x;
    const int a = g.a, b = g.b, c = g.c, n = g.n, nb = g.nb;
    z* Al = A + (size_t)leaf * n * n;
    for (long long e = threadIdx.x; e < (long long)n * n; e += blockDim.x) Al[e] = zmk(0.0, 0.0);
    __syncthreads();
    const double h[3] = {hh[3 * leaf], hh[3 * leaf + 1], hh[3 * leaf + 2]};
    // one thread owns a row: its entries are accumulated in FD_matrix_row's order
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        if (r < nb) {
            int p1, p2, ax;
            bnd3(r, a, b, c, p1, p2, ax);
            const double hn = h[ax];
            Al[r + (size_t)r * n] = zadd(zmk(0.0, g.kb), zmk((8.0 / 3.0) / hn, 0.0));
            Al[r + (size_t)p1 * n] = zmk(-3.0 / hn, 0.0);
            Al[r + (size_t)p2 * n] = zmk((1.0 / 3.0) / hn, 0.0);
        } else {
            int gi, gj, gk;
            grid3(r, a, b, c, gi, gj, gk);
            const int gg[3] = {gi, gj, gk}, sh[3] = {a, b, c};
            z diag = kv[(size_t)leaf * (a * b * c) + (r - nb)];
            for (int d = 0; d < 3; ++d) {
                double w0 = 1.0, w1 = -2.0, w2 = 1.0;
                if (gg[d] == 1) { w0 = 8.0 / 3.0; w1 = -4.0; w2 = 4.0 / 3.0; }
                else if (gg[d] == sh[d]) { w0 = 4.0 / 3.0; w1 = -4.0; w2 = 8.0 / 3.0; }
                const double h2 = h[d] * h[d];
                diag = zadd(diag, zmk(w1 / h2, 0.0));
                const int up = lin3(gi + (d == 0), gj + (d == 1), gk + (d == 2), a, b, c);
                const int dn = lin3(gi - (d == 0), gj - (d == 1), gk - (d == 2), a, b, c);
                Al[r + (size_t)up * n] = zadd(Al[r + (size_t)up * n], zmk(w2 / h2, 0.0));
                Al[r + (size_t)dn * n] = zadd(Al[r + (size_t)dn * n], zmk(w0 / h2, 0.0));
            }
            Al[r + (size_t)r * n] = diag;
        }
    }
}

// Y = R A^-1 (nb x n, ld nb): the face rows of the inverse turned into outgoing Robin data.
__global__ void __launch_bounds__(256) leaf3_rtr_kernel(Leaf3Geom g, const double* __restrict__ hh,
                                                        const z* __restrict__ Ainv, z* Y) {
    const int leaf = blockIdx.x;
    const int n = g.n, nb = g.nb;
    const z* X = Ainv + (size_t)leaf * n * n;
    z* Yl = Y + (size_t)leaf * nb * n;
    const double h[3] = {hh[3 * leaf], hh[3 * leaf + 1], hh[3 * leaf + 2]};
    const z sigma = zmk(0.0, -g.kb);
    for (long long e = threadIdx.x; e < (long long)nb * n; e += blockDim.x) {
        const int r = (int)(e % nb), col = (int)(e / nb);
        int p1, p2, ax;
        bnd3(r, g.a, g.b, g.c, p1, p2, ax);
        const double hn = h[ax];
        const z x0 = X[r + (size_t)col * n];
        z v = zadd(zmul(sigma, x0), zscale((8.0 / 3.0) / hn, x0));
        v = zadd(v, zscale(-3.0 / hn, X[p1 + (size_t)col * n]));
        v = zadd(v, zscale((1.0 / 3.0) / hn, X[p2 + (size_t)col * n]));
        Yl[e] = v;
    }
}

cudaError_t leaf3_assemble(const Leaf3Geom& g, int nleaves, const double* hh, const z* kv, z* A, cudaStream_t s) {
    leaf3_assemble_kernel<<<nleaves, 256, 0, s>>>(g, hh, kv, A);
    note_launch();
    return cudaGetLastError();
}

cudaError_t leaf3_rtr(const Leaf3Geom& g, int nleaves, const double* hh, const z* Ainv, z* Y, cudaStream_t s) {
    leaf3_rtr_kernel<<<nleaves, 256, 0, s>>>(g, hh, Ainv, Y);
    note_launch();
    return cudaGetLastError();
}

}  // namespace rb
