// rb_kernels.h -- internal launch interface of the CUDA kernels (not part of the C-ABI).
#pragma once
#include <cuda_runtime.h>
#include "rb_common.cuh"

namespace rb {

// ---- launch accounting --------------------------------------------------------------------------
void note_launch();
long long launch_count();
// message returned by rb_last_error(NULL) on this thread
void set_thread_error(const char* msg);

// ---- batched GEMM ---------------------------------------------------------------------------------
cudaError_t launch_gemm_batch(const GemmBatch& b, cudaStream_t s);
// Chooses split-K for a fixed-order batch (sets ksplit, kchunk, pstride) and returns the
// workspace it needs in complex elements (0: no split); the caller sets b.work.
long long gemm_plan_split(GemmBatch& b);
// stage-timer name of the kernel a batch runs on: "zgemm_tc" (the contiguous-k tensor-core tile
// of the large merges), "zgemm_tc_small" (the other tensor-core factor tiles), "zgemm_tc_fixed"
// (the solve's fixed-order tensor-core tile) or "zgemm_dfma" (DFMA register tiles)
const char* gemm_stage_name(const GemmBatch& b);

// ---- batched Gauss-Jordan inversion (in place, partial pivoting by |re|+|im|) ----------------------
struct GJDesc {
    z* A;          // m x m, column-major
    long long ld;
    int* ipiv;     // m
    z* Zb;         // workspace: the resident path's flag words (gj_workspace_elems)
};
constexpr int GJ_SMALL_MAX = 64;       // largest matrix the whole-matrix kernel holds
constexpr int GJ_BLOCKED_MIN = 33;     // from this size on: resident (else blocked) path
int gj_panel_width(int m);                         // nb of the blocked path (0 for the small path)
long long gj_workspace_elems(int m);               // complex elements of Zb per matrix
// work: the count descriptors' Zb areas, contiguous (count * gj_workspace_elems(m) elements)
cudaError_t gj_invert_batch(const GJDesc* d_desc, int count, int m, void* work, int* d_status, cudaStream_t s);

// ---- leaf stage ---------------------------------------------------------------------------------------
struct LeafGeom {
    int a, b;          // interior grid
    int nb, n;         // boundary points, unknowns
    double kb;         // solve_opts%kb
};
// Structured leaf factor (rb_leaf.cu): per leaf the inverted diagonal blocks Sig_j^-1 of the
// block-tridiagonal interior Schur complement (b blocks of a x a, at sinv + leaf*b*a*a) and
// Y = R A^-1 (nb x n, ld nb, at Y + leaf*nb*n); k: nleaves*a*b potential samples.
size_t leaf_block_factor_smem(const LeafGeom& g);
cudaError_t leaf_block_factor(const LeafGeom& g, int nleaves, const double* h, const z* k, z* sinv, z* Y,
                              int* status, cudaStream_t s);
// Structured leaf solve: u = A^-1 [g; f] into sol [rhs][leaf][n]; f is [rhs][leaf][a*b] (may be
// null for zero sources), gb is [leaf][rhs][nb].
cudaError_t leaf_block_solve(const LeafGeom& g, int nleaves, int nrhs, const double* h, const z* f, const z* gb,
                             const z* sinv, z* sol, cudaStream_t s);

// ---- merge helpers -------------------------------------------------------------------------------------
struct ChildStore {
    const z* rtr;      // node 0's Robin-to-Robin matrix
    long long stride;  // elements between consecutive nodes
    long long ld;      // leading dimension
};
// D = zeta*I - T2_ii for every parent node (child2 = 2*node+1), into dst + node*m*m.
cudaError_t merge_form_d(ChildStore c, int nnodes, int m, int o2, z zeta, z* dst, cudaStream_t s);
// S = zeta*I - T1_ii - nu^2 * Dinv for every parent node (child1 = 2*node).
cudaError_t merge_form_s(ChildStore c, int nnodes, int m, int o1, z zeta, z nu, const z* dinv, z* dst,
                         cudaStream_t s);
// K = nu^2 I for every node, into dst + node*m*m.
cudaError_t merge_form_k(int nnodes, int m, z nu, z* dst, cudaStream_t s);

// ---- device-side sampling and check_solution (rb_sample.cu) -------------------------------------------
// pts: n points (x, y, z) as rb_tree_sample_points lists them; outputs complex128
cudaError_t sample_bump(const double* pts, long long n, double kb, double delta, double w, int nbumps,
                        const double* d_bumps, z* out, cudaStream_t s);
cudaError_t sample_point_sources(const double* pts, long long n, int nrhs, const double* d_par, z* f, cudaStream_t s);
cudaError_t sample_plane_waves(const double* pts, int nb, int ra, int rb, const double* dom4, int nrhs,
                               const double* d_par, z* g, cudaStream_t s);
cudaError_t check_solution(const z* u, const z* ue, int nleaves, int n, int norm, int rel, double* err,
                           cudaStream_t s);

// ---- sweep helpers --------------------------------------------------------------------------------------
// children's g on their non-interface faces from the parent's g (backward sweep):
// g_child[phys(t)] = g_parent[pmap[t]] for both children, every node and RHS.
cudaError_t sweep_scatter_down(int nnodes, int nrhs, int nbp, int nbc, int m, int o1, int o2, int n1,
                               int n2, const int* pmap1, const int* pmap2, const z* gpar, z* gchild,
                               cudaStream_t s);

}  // namespace rb
