// rb_kernels.h -- internal launch interface of the CUDA kernels (not part of the C-ABI).
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <mutex>
#include "rb_common.cuh"

namespace rb {

// ---- per-device kernel attributes -----------------------------------------------------------------
// A kernel's dynamic shared-memory limit (and carveout preference) is a setting of the current
// device, not of the process.  Each launch site keeps one cache: the largest limit it has set on
// each device, so that a handle on a second device (or a second host thread) sets it there too.
struct DeviceAttrCache {
    std::mutex mu;
    std::atomic<size_t> set[128] = {};
};
template <class K>
inline cudaError_t ensure_smem_attr(K kern, size_t bytes, DeviceAttrCache& c, bool max_carveout = false) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const bool cached = dev >= 0 && dev < 128;
    if (cached && c.set[dev].load(std::memory_order_acquire) >= bytes) return cudaSuccess;
    std::lock_guard<std::mutex> lk(c.mu);
    const size_t want = cached ? std::max(bytes, c.set[dev].load(std::memory_order_relaxed)) : bytes;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)want);
    if (e != cudaSuccess) return e;
    if (max_carveout) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
    }
    if (cached) c.set[dev].store(want, std::memory_order_release);
    return cudaSuccess;
}

// ---- launch accounting --------------------------------------------------------------------------
void note_launch();
long long launch_count();
// message returned by rb_last_error(NULL) on this thread
void set_thread_error(const char* msg);

// ---- device status word ----------------------------------------------------------------------------
// Bits a kernel ORs into a handle's status word (read after a factor or solve).
constexpr int RB_STATUS_ZERO_PIVOT = 1;     // a leaf block or interface inverse met a zero pivot
constexpr int RB_STATUS_GJ_TIMEOUT = 2;     // a resident Gauss-Jordan CTA gave up waiting for a panel
constexpr int RB_TC5_TIMEOUT = 4;           // a tensor-core GEMM CTA gave up waiting on an mbarrier

// ---- batched GEMM ---------------------------------------------------------------------------------
cudaError_t launch_gemm_batch(const GemmBatch& b, cudaStream_t s);
// The same batch on the tcgen05 tensor cores (rb_gemm_tc5.cu), for the mixed-precision levels, in
// one of two arithmetics (b.t5_engine): split TF32 with FP32 accumulation (~1e-7 of
// max|A| max|B| k), or the default, int8 digit slices of row- and column-scaled operands with
// exact int32 accumulation (~1e-10 of that scale).  status: device word for RB_TC5_TIMEOUT.
cudaError_t launch_gemm_tc5(const GemmBatch& b, int* status, cudaStream_t s);
constexpr int TC5_ENGINE_TF32X3 = 0;
constexpr int TC5_ENGINE_INT8 = 1;
// the engine a batch runs on: its own t5_engine, else the process default (RB_MIXED_ENGINE =
// "tf32x3" or "int8", read once; int8 when unset)
int tc5_engine(const GemmBatch& b);
int tc5_tile_n(const GemmBatch& b);
// Bytes of operand planes launch_gemm_tc5 needs for this batch (b.t5_planes).
size_t tc5_plane_bytes(const GemmBatch& b);
// Engines (tile shapes) of the FP64 launcher that can run a non-fixed-order batch, for the
// autotuner: writes up to 8 engine ids to out (a batch's `engine` field takes one) and returns
// the count.  gemm_engine_name gives each a stage-timer name.
int gemm_engine_candidates(const GemmBatch& b, int* out);
const char* gemm_engine_name(int engine);
// Chooses split-K of a batch on the tcgen05 kernel (sets t5_ksplit, t5_kchunk, t5_pstride; from
// count, m and k only) and returns the workspace it needs in complex elements (0: no split).
long long gemm_plan_split_tc5(GemmBatch& b);
// The same for a factor stage: only stages with fewer 128-row tiles than SMs are split.
long long gemm_plan_split_tc5_factor(GemmBatch& b);
// Adds the split ranges' raw sums in range order and applies the problem's epilogue (alpha, beta,
// C, output maps): the second pass of every split-K GEMM.
cudaError_t launch_gemm_reduce(const GemmBatch& b, int ksplit, long long pstride, cudaStream_t s);
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

// Dense 3D leaf (rb_leaf3d.cu): A (n x n, column-major, at A + leaf*n*n) from the leaf's spacings
// hh (3 per leaf) and potential kv (a*b*c per leaf, x fastest); Y = R A^-1 (nb x n, ld nb) from
// A^-1 in place of A.
struct Leaf3Geom {
    int a, b, c;       // interior grid
    int nb, n;         // boundary points 2(bc+ac+ab), unknowns nb + abc
    double kb;
};
cudaError_t leaf3_assemble(const Leaf3Geom& g, int nleaves, const double* hh, const z* kv, z* A, cudaStream_t s);
cudaError_t leaf3_rtr(const Leaf3Geom& g, int nleaves, const double* hh, const z* Ainv, z* Y, cudaStream_t s);

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
// The three K-form merge inputs of one node of any tree and level (a forest's batched merge).
struct MergeFormDesc {
    const z* t1;       // child1's Robin-to-Robin matrix
    const z* t2;       // child2's
    long long ld;
    int m, o1, o2, pad;
    z zeta, nu2;
    z* a2;             // zeta I - T2_ii
    z* a1;             // zeta I - T1_ii
    z* k;              // nu^2 I
};
cudaError_t merge_form_kform_batch(const MergeFormDesc* d_descs, int count, int max_m, cudaStream_t s);

// ---- device-side sampling and check_solution (rb_sample.cu) -------------------------------------------
// pts: n points (x, y, z) as rb_tree_sample_points lists them; outputs complex128
cudaError_t sample_bump(const double* pts, long long n, double kb, double delta, double w, int nbumps,
                        const double* d_bumps, z* out, cudaStream_t s);
cudaError_t sample_point_sources(const double* pts, long long n, int nrhs, const double* d_par, z* f, cudaStream_t s);
cudaError_t sample_plane_waves(const double* pts, int nb, int ra, int rb, const double* dom4, int nrhs,
                               const double* d_par, z* g, cudaStream_t s);
cudaError_t check_solution(const z* u, const z* ue, int nleaves, int n, int norm, int rel, double* err,
                           cudaStream_t s);

// ---- iterative refinement of the mixed-precision solve (rb_refine.cu) ------------------------------------
struct RefineGeom {
    int a, b;          // leaf grid
    int nleaves;
    int root_nb;       // boundary points of the whole domain
    double kb;         // solve_opts%kb (FD boundary rows)
    z zeta, nu;        // transmission coefficients of the merge (bndry_params)
};
// r <- r - A d for the global FD system, in place: interior rows in f [rhs][leaf][ab], domain
// boundary rows in groot [rhs][root_nb], interface rows in ri [rhs][leaf][nb] (zero before when
// first).  bclass[leaf*nb + r]: root position (>= 0) or -1 - (neighbour's leaf*nb + row).
// rnorm[rhs] accumulates max |r| (|re| + |im|) when non-null.
cudaError_t fd_residual(const RefineGeom& g, int nrhs, const z* d, z* f, z* groot, z* ri, const z* kv,
                        const double* hh, const int* bclass, bool first, double* rnorm, cudaStream_t s);
// hbuf of level l's children -= ri at the interface points listed in rows (nnodes*2*m leaf rows)
cudaError_t iface_inject(int nnodes, int m, int nbc, int o1, int o2, int nrhs, int leaf_rows, const int* rows,
                         const z* ri, z* hbuf, cudaStream_t s);
// x += dx; per right-hand side max |x| into xnorm and max |dx| into dnorm (accumulated)
cudaError_t refine_update(z* x, const z* dx, long long per, int nrhs, double* xnorm, double* dnorm, cudaStream_t s);

// ---- sweep helpers --------------------------------------------------------------------------------------
// children's g on their non-interface faces from the parent's g (backward sweep):
// g_child[phys(t)] = g_parent[pmap[t]] for both children, every node and RHS.
cudaError_t sweep_scatter_down(int nnodes, int nrhs, int nbp, int nbc, int m, int o1, int o2, int n1,
                               int n2, const int* pmap1, const int* pmap2, const z* gpar, z* gchild,
                               cudaStream_t s);

}  // namespace rb
