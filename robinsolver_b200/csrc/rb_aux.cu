// rb_aux.cu -- merge and sweep helper kernels for sm_100a.
//
// The merge helpers form the interface matrices D and S of compute_RTR; the sweep helpers move
// boundary data between a node and its children.
#include <algorithm>

#include "rb_kernels.h"

namespace rb {

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

// K = nu^2 I for every node (the GEMM K -= A2 A1 then completes K = nu^2 I - A2 A1)
__global__ void merge_form_k_kernel(int m, z nu2, z* __restrict__ dst) {
    const int node = blockIdx.y;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= m * m) return;
    const int r = idx % m, q = idx / m;
    dst[(long long)node * m * m + idx] = r == q ? nu2 : zmk(0.0, 0.0);
}

cudaError_t merge_form_k(int nnodes, int m, z nu, z* dst, cudaStream_t s) {
    dim3 grid((m * m + 255) / 256, nnodes);
    merge_form_k_kernel<<<grid, 256, 0, s>>>(m, zmul(nu, nu), dst);
    note_launch();
    return cudaGetLastError();
}

// One node of a batched K-form merge (several trees, several levels): A2 = zeta I - T2_ii,
// A1 = zeta I - T1_ii, K = nu^2 I, each m x m.
__global__ void merge_form_kform_kernel(const MergeFormDesc* __restrict__ descs) {
    const MergeFormDesc d = descs[blockIdx.y];
    const int m = d.m;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < m * m; idx += gridDim.x * blockDim.x) {
        const int r = idx % m, q = idx / m;
        z a2 = zneg(d.t2[(d.o2 + r) + (long long)(d.o2 + q) * d.ld]);
        z a1 = zneg(d.t1[(d.o1 + r) + (long long)(d.o1 + q) * d.ld]);
        if (r == q) {
            a2 = zadd(a2, d.zeta);
            a1 = zadd(a1, d.zeta);
        }
        d.a2[idx] = a2;
        d.a1[idx] = a1;
        d.k[idx] = r == q ? d.nu2 : zmk(0.0, 0.0);
    }
}

cudaError_t merge_form_kform_batch(const MergeFormDesc* d_descs, int count, int max_m, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    if (count > 65535) return cudaErrorInvalidValue;
    const int bx = std::min((max_m * max_m + 255) / 256, 64);
    merge_form_kform_kernel<<<dim3(bx, count), 256, 0, s>>>(d_descs);
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

}  // namespace rb
