// rb_sample.cu -- device-side sampling of the standard potential and right-hand sides, and
// check_solution's per-leaf error norms, for sm_100a.
//
// The reference evaluates elliptic_operator%k, elliptic_rhs%f and bndry_rhs%g_face on the host,
// one point at a time (fd_module.f90:136-145, 427-431, 636-651).  For the three families of the
// synthetic problems (a Gaussian-bump potential, Gaussian point sources, plane waves through
// the impedance boundary) these kernels evaluate the same formulas on the device at the very
// points rb_tree_sample_points lists, so a right-hand side never crosses PCIe.  Products and
// sums that form an exponent are rounded one by one (__dmul_rn/__dadd_rn: no contraction into
// FMA), as the host computes them; exp, cos and sin are CUDA's.
//
// check_solution (robin_output_module.f90:84-134) compares each leaf's solution vector with the
// exact solution sampled at the same points and reports one 1-, 2- or max-norm per leaf,
// absolute or relative; here the solution never leaves the device.
#include "rb_kernels.h"

namespace rb {

// k = kb (1 + 0.3 sum_j a_j exp(-|x - c_j|^2 / (2 w^2))) + i delta kb;  bumps: (cx, cy, a) per bump
__global__ void sample_bump_kernel(const double* __restrict__ pts, long long n, double kb, double delta, double w,
                                   int nbumps, const double* __restrict__ bumps, z* __restrict__ out) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double x = pts[3 * p], y = pts[3 * p + 1];
    const double w2 = __dmul_rn(__dmul_rn(2.0, w), w);
    double s = 0.0;
    for (int j = 0; j < nbumps; ++j) {
        const double dx = __dadd_rn(x, -bumps[3 * j]), dy = __dadd_rn(y, -bumps[3 * j + 1]);
        const double r2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
        s = __dadd_rn(s, __dmul_rn(bumps[3 * j + 2], exp(-r2 / w2)));
    }
    out[p] = zmk(__dmul_rn(kb, __dadd_rn(1.0, __dmul_rn(0.3, s))), __dmul_rn(delta, kb));
}

// f = exp(-|x - x0|^2 / (2 w^2)) per right-hand side; par: (x0, y0, w) per RHS
__global__ void sample_point_source_kernel(const double* __restrict__ pts, long long n,
                                           const double* __restrict__ par, z* __restrict__ f) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (p >= n) return;
    const double x0 = par[3 * r], y0 = par[3 * r + 1], w = par[3 * r + 2];
    const double dx = __dadd_rn(pts[3 * p], -x0), dy = __dadd_rn(pts[3 * p + 1], -y0);
    const double r2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
    f[(long long)r * n + p] = zmk(exp(-r2 / __dmul_rn(__dmul_rn(2.0, w), w)), 0.0);
}

// g = i kb (d.n - 1) exp(i kb d.x) on the boundary points (faces x1 x2 y1 y2 of rb, rb, ra, ra
// points, face-local coordinate in column 0); par: (kb, dx, dy) per RHS; dom: x lo, x hi, y lo, y hi
__global__ void sample_plane_wave_kernel(const double* __restrict__ pts, int nb, int ra, int rb, double4 dom,
                                         const double* __restrict__ par, z* __restrict__ g) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (p >= nb) return;
    const double kb = par[3 * r], ddx = par[3 * r + 1], ddy = par[3 * r + 2];
    const double t = pts[3 * p];
    double x, y, nx = 0.0, ny = 0.0;
    if (p < rb) { x = dom.x; y = t; nx = -1.0; }
    else if (p < 2 * rb) { x = dom.y; y = t; nx = 1.0; }
    else if (p < 2 * rb + ra) { x = t; y = dom.z; ny = -1.0; }
    else { x = t; y = dom.w; ny = 1.0; }
    const double dn = __dadd_rn(__dmul_rn(ddx, nx), __dmul_rn(ddy, ny));
    const double ph = __dmul_rn(kb, __dadd_rn(__dmul_rn(ddx, x), __dmul_rn(ddy, y)));
    double sn, cs;
    sincos(ph, &sn, &cs);
    // i kb (dn - 1) (cos + i sin)
    const double c = __dmul_rn(kb, __dadd_rn(dn, -1.0));
    g[(long long)r * nb + p] = zmk(-__dmul_rn(c, sn), __dmul_rn(c, cs));
}

// one block per leaf: norm of u - u_exact (or of (u - u_exact) / u_exact) over the leaf's points;
// norm 1: sum, 2: sqrt of the sum of squares, otherwise the maximum
__global__ void __launch_bounds__(256) check_solution_kernel(const z* __restrict__ u, const z* __restrict__ ue, int n,
                                                             int norm, int rel, double* __restrict__ err) {
    __shared__ double red[256];
    const int leaf = blockIdx.x;
    const z* ul = u + (long long)leaf * n;
    const z* el = ue + (long long)leaf * n;
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        z d = zsub(ul[i], el[i]);
        if (rel) {
            const z q = zrcp(el[i]);
            d = zmul(d, q);
        }
        const double a = hypot(d.x, d.y);
        if (norm == 1) acc += a;
        else if (norm == 2) acc += a * a;
        else acc = fmax(acc, a);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            const double b = red[threadIdx.x + o];
            red[threadIdx.x] = (norm == 1 || norm == 2) ? red[threadIdx.x] + b : fmax(red[threadIdx.x], b);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) err[leaf] = norm == 2 ? sqrt(red[0]) : red[0];
}

cudaError_t sample_bump(const double* pts, long long n, double kb, double delta, double w, int nbumps,
                        const double* d_bumps, z* out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    sample_bump_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pts, n, kb, delta, w, nbumps, d_bumps, out);
    note_launch();
    return cudaGetLastError();
}

cudaError_t sample_point_sources(const double* pts, long long n, int nrhs, const double* d_par, z* f, cudaStream_t s) {
    if (n <= 0 || nrhs <= 0) return cudaSuccess;
    sample_point_source_kernel<<<dim3((unsigned)((n + 255) / 256), nrhs), 256, 0, s>>>(pts, n, d_par, f);
    note_launch();
    return cudaGetLastError();
}

cudaError_t sample_plane_waves(const double* pts, int nb, int ra, int rb, const double* dom4, int nrhs,
                               const double* d_par, z* g, cudaStream_t s) {
    if (nb <= 0 || nrhs <= 0) return cudaSuccess;
    const double4 dom = make_double4(dom4[0], dom4[1], dom4[2], dom4[3]);
    sample_plane_wave_kernel<<<dim3((nb + 255) / 256, nrhs), 256, 0, s>>>(pts, nb, ra, rb, dom, d_par, g);
    note_launch();
    return cudaGetLastError();
}

cudaError_t check_solution(const z* u, const z* ue, int nleaves, int n, int norm, int rel, double* err,
                           cudaStream_t s) {
    if (nleaves <= 0) return cudaSuccess;
    check_solution_kernel<<<nleaves, 256, 0, s>>>(u, ue, n, norm, rel, err);
    note_launch();
    return cudaGetLastError();
}

}  // namespace rb
