// rb_tree_impl.hpp -- the state of a tree handle (struct rb_tree), shared by the translation units
// that drive handles directly: rb_tree.cpp (the C-ABI of one tree) and rb_forest.cpp (several trees
// factored in one level-synchronous schedule).  Not part of the C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "robin_b200.h"
#include "rb_kernels.h"
#include "rb_plan.hpp"

namespace rb {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct GJBatch {
    GJDesc* d_desc = nullptr;
    int count = 0;
    int m = 0;
};

// The solve's launch plan for one RHS count: its descriptor batches, their device arrays (and
// split-K workspace), and its captured graph.  A tree keeps a few of them, so that solves whose
// RHS counts change from call to call (a serving loop's batches) reuse them instead of uploading
// descriptors and capturing a graph again.
struct SolveSet {
    int nrhs = 0;
    GemmBatch sL0, sLg, sLf, sR1;
    std::vector<GemmBatch> sF12, sF3, sF4, sF5, sBY;
    std::vector<DevBuf> bufs;
    cudaGraphExec_t gx = nullptr;
    long long gx_launches = 0;
    int runs = 0;
    unsigned long long used = 0;
};

struct StageTimer {
    const char* name;
    double flops;
    int ev;          // index of the start event in the pool (end = ev + 1)
};

}  // namespace rb

// the C-ABI declares struct rb_tree at global scope; its members are this library's types
using namespace rb;

struct rb_tree {
    rb_geom geom;
    Plan P;
    std::string err;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;      // runs one merge GEMM per level beside the level's inversion
    cudaStream_t stream3 = nullptr;      // host -> device copies of the inputs, beside running work
    // rb_get_solution_async: device -> host copies of solutions on their own stream, behind the solve
    // that wrote them; the next solve waits for ev_d2h before it writes the solution buffer
    cudaStream_t stream5 = nullptr;
    cudaEvent_t ev_d2h = nullptr;
    bool d2h_pending = false;
    cudaEvent_t ev_copy = nullptr;
    // RB_FLAG_ASYNC_FACTOR: rb_tree_factor returns once the factor is enqueued; its completion,
    // time and status are taken by the next call that needs them (settle_factor)
    bool async_factor = false;
    bool factor_pending = false;
    int* h_status = nullptr;             // pinned: [0] the factor's status word after the factor,
                                         // [1] the same word as the overlapped solve saw it
    bool solve_overlapped = false;       // the last solve ran beside its factor (on stream3)
    std::vector<cudaEvent_t> ev_fork, ev_join;
    // factor progress for a solve that overlaps it: [l] after level l's inversion, [L] after the leaves
    std::vector<cudaEvent_t> ev_lvl;
    cudaEvent_t ev_root_forms = nullptr; // the root's A2 (D) is formed, after level 1's maps
    bool factor_deferred = false;        // RB_FLAG_ASYNC_FACTOR: potential copied, factor not launched
    // device-side sampling and check_solution: rb_tree_sample_points' points, cached on first use
    double* d_pts[3] = {nullptr, nullptr, nullptr};     // potential, source, boundary
    double* d_par = nullptr;
    size_t par_cap = 0;
    double* d_err = nullptr;
    z* d_uex = nullptr;
    int device = 0;
    bool factored = false;
    double f_time = 0.0, s_time = 0.0;
    z zeta, nu;
    int64_t budget = 0;
    std::vector<DevBuf> bufs;        // every allocation, for the budget and destroy
    int64_t held = 0;
    bool verbose = false;
    bool skip_root = false;

    // persistent factor storage
    double* d_h = nullptr;
    z* d_k = nullptr;
    z* leaf_sinv = nullptr;          // 2D: the leaves' Sig_j^-1 blocks; 3D: each leaf's dense A^-1
    z* leaf_Y = nullptr;
    GJBatch gj_leaf;                 // 3D: the leaves' Gauss-Jordan inversions (A^-1 in leaf_sinv)
    int* leaf_ipiv = nullptr;
    z* leaf_gjwork = nullptr;
    std::vector<z*> rtr;             // per level < L
    std::vector<z*> dinv, sinv;      // per level < L: inv(D), inv(S); in the K form A2, A1
    // K form of the interface solve (nu not small): one inversion per node instead of two
    bool kform = false;
    std::vector<z*> kinv;            // per level < L, K form only
    std::vector<int*> d_pmap1, d_pmap2;
    std::vector<int*> d_pmapc;       // per level < L: pmap1 then pmap2 (the columns of Y1 and Y2)
    int* d_status = nullptr;
    // per level < L: [Y1; Y2] = M^-1 blockdiag(T1_iN, T2_iN), nnodes x m x (n1 + n2) each; the
    // backward sweep below the root applies them to the node's incoming data
    std::vector<z*> Y1, Y2;
    z* gj_work = nullptr;
    int* gj_ipiv = nullptr;
    // factor launch batches
    std::vector<GJBatch> gj_d, gj_s, gj_k;
    std::vector<GemmBatch> fK, fM1, fM2, fM3, fM4;
    // Level-pipelined FP64 factor: level l's parent map split by rows into the rows on the face
    // its parent merges across (fM4F: all the parent's interface solve reads) and the others
    // (fM4N), so that the parent level's forms, K and inversion run beside fM4N (levels 1..L-1)
    std::vector<GemmBatch> fM4F, fM4N;
    cudaStream_t stream4 = nullptr;      // the pipelined factor's B1 product beside the inversion
    std::vector<cudaEvent_t> ev_face, ev_rest, ev_d, ev_m1, ev_m3;   // per level
    cudaEvent_t ev_root_gj = nullptr;
    bool factor_was_pipelined = false;   // the last factor ran the pipelined schedule
    bool factor_ready = false;

    // solve storage
    int cap_rhs = 0;                 // capacity of the solve buffers
    int built_rhs = 0;               // nrhs the solve batches were built for
    int nrhs = 0;                    // RHS held from the last solve
    z* d_f = nullptr;
    std::vector<z*> hbuf, gbuf;      // per level 0..L
    z* tmp = nullptr;
    z* sol = nullptr;
    GemmBatch sL0;
    GemmBatch sLg, sLf;              // 3D leaf solve: u = A^-1(:, :nb) g, then u += A^-1(:, nb:) f
    std::vector<GemmBatch> sF12, sF3, sF4, sF5, sBY;
    GemmBatch sR1;                   // root: x_i = h_i + T_iN g_N (no K^-1 needed)
    std::vector<DevBuf> solve_bufs;
    std::vector<DevBuf> solve_desc_bufs;     // the current RHS count's descriptor arrays and workspace
    std::vector<SolveSet> solve_sets;        // other RHS counts' plans, least recently used evicted
    unsigned long long solve_clock = 0;
    unsigned char* solve_planes = nullptr;   // tcgen05 operand planes of the solve (mixed, tc5 sweeps)
    size_t solve_planes_bytes = 0;

    // timing: 0 off, 1 per stage, 2 per launch
    int timing = 0;
    struct StageTime { std::string name; double ms; double flops; };
    std::vector<StageTime> stage_ms;
    std::vector<StageTimer> timers;
    std::vector<cudaEvent_t> ev_pool;
    int ev_used = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    int64_t factor_launches = 0, solve_launches = 0;

    // RB_PREC_MIXED: the GEMMs of the merge levels l >= 2 whose interface is at least one
    // tensor-core tile tall (m >= 128) run on the tcgen05 split-TF32 kernel (~1e-6 relative);
    // the top two levels, the interface inverses, the leaves and the FD residual stay FP64, and
    // the solve refines every right-hand side against the FP64 residual to refine_tol
    int prec = RB_PREC_FP64;          // precision of the current factorization
    bool mixed_int8_top = false;      // RB_FLAG_MIXED_INT8_TOP
    int gx_factor_prec = -1;          // precision the captured factor graph was recorded with
    double refine_tol = 1e-10;
    int refine_maxit = 8;
    int refine_iters = 0;             // corrections the last solve applied
    double refine_rho = 0.0;          // largest contraction factor seen
    double refine_est = 0.0;          // estimated relative error after the last correction
    double refine_res = 0.0;          // max |r| / max |x| of the last residual
    std::vector<int> h_bclass;        // leaf boundary row -> root position or -1 - neighbour row
    std::vector<std::vector<int>> h_ifrows;   // per level: interface points -> leaf boundary rows
    int* d_bclass = nullptr;
    std::vector<int*> d_ifrows;
    int refine_cap = 0;
    bool mixed_plan = false;          // split-K plans and workspaces of the tcgen05 factor stages
    std::vector<DevBuf> mixed_bufs;
    z* dsol = nullptr;                // the correction of the current refinement step
    z* d_ri = nullptr;                // interface rows of the residual [rhs][leaf][nb]
    double* d_norms = nullptr;        // [0, k) max|r|, [k, 2k) max|x|, [2k, 3k) max|dx|
    double* h_norms = nullptr;
    std::vector<DevBuf> refine_bufs;

    // CUDA graphs: the factor and solve launch sequences are fixed per tree (and per RHS count),
    // so after one direct run each is captured once and replayed
    bool graphs = true;
    int factor_runs = 0;
    cudaGraphExec_t gx_factor = nullptr;
    long long gx_factor_launches = 0;
    int solve_runs = 0;
    cudaGraphExec_t gx_solve = nullptr;
    int gx_solve_rhs = 0;
    long long gx_solve_launches = 0;
};

