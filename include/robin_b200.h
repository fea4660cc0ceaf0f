/*
 * robin_b200.h -- C-ABI of the B200 hierarchical Poincare-Steklov (HPS) factor/solve.
 *
 * Drop-in boundary for robinsolver's hot path.  Every entry point takes plain
 * pointers and sizes; complex numbers are interleaved (re, im) double pairs, the
 * layout of C99 `double _Complex` and Fortran `complex(c_double_complex)`.
 * Arrays handed in by the caller are read before the call returns (host arrays)
 * or are device arrays the caller keeps alive until the call returns.
 *
 * The reference's callbacks (elliptic_operator%k, elliptic_rhs%f, bndry_rhs%g_face)
 * are evaluated by the caller on the host at points this library reports
 * (rb_tree_sample_points); the library never calls back into user code.
 *
 * Status codes: 0 on success, a negative RB_ERR_* value on failure; the message of
 * the last failure on a handle is returned by rb_last_error(handle), and
 * rb_last_error(NULL) reports the last failure of rb_tree_create (or of
 * rb_leaf_rtr_noalloc) on this thread.
 * The reference stops the process instead ("stop '<message>'"); the messages below
 * carry the reference's wording where one exists.
 *
 * Threading: one host thread at a time per handle.  Different handles are
 * independent.  All device work of a handle runs on the handle's CUDA stream.
 */
#ifndef ROBIN_B200_H
#define ROBIN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------------------------- */
#define RB_OK                  0
#define RB_ERR_INVALID        -1  /* bad argument (null pointer, size, index)                        */
#define RB_ERR_DOMAIN         -2  /* "Invalid operator domain format." / "Dimension must be 2 or 3."  */
#define RB_ERR_BNDRY_PARAMS   -3  /* "Boundary parameter matrix is nearly singular."                  */
#define RB_ERR_NOT_FACTORED   -4  /* "Robin Tree must be factored first."                            */
#define RB_ERR_DIM_MISMATCH   -5  /* "Dimensions of Robin Tree and RHS do not match."                */
#define RB_ERR_GEOMETRY       -6  /* "Interface sizes of node children do not match." (non-uniform)   */
#define RB_ERR_UNSUPPORTED    -7  /* a valid request this build does not implement (interfaces over
                                     1024 points, a mixed-precision or forest factor in 3D, ...)   */
#define RB_ERR_CUDA           -8  /* CUDA runtime failure (message carries cudaGetErrorString)        */
#define RB_ERR_OUT_OF_MEMORY  -9  /* device allocation refused or over the handle's byte budget       */
#define RB_ERR_NUMERIC       -10  /* zero pivot / non-finite value met during the factorization       */
#define RB_ERR_NO_SOLUTION   -11  /* get_solution before any solve, or irhs out of range              */

/* ---- precision modes for rb_tree_factor ----------------------------------------------------- */
#define RB_PREC_FP64  0           /* every operation in complex128                                    */
#define RB_PREC_MIXED 1           /* merge levels l >= 2 with interfaces of >= 128 points: GEMMs on the
                                     tcgen05 tensor cores in split TF32 (FP32 accumulation, ~1e-6
                                     relative); the top two levels, the interface inverses, the leaves
                                     and the FD residual in FP64; every solve refined against the FP64
                                     residual of the global FD system to the tree's tolerance
                                     (rb_tree_set_refinement, default 1e-10 relative)                  */

/* ---- sample-point kinds for rb_tree_sample_points ------------------------------------------- */
#define RB_POINTS_POTENTIAL 0     /* interior cell centres where elliptic_operator%k is sampled       */
#define RB_POINTS_SOURCE    1     /* interior cell centres where elliptic_rhs%f is sampled            */
#define RB_POINTS_BOUNDARY  2     /* face-local coordinates where bndry_rhs%g_face is sampled         */
#define RB_POINTS_SOLUTION  3     /* every point of every leaf's u vector (check_solution's points)   */

/* ---- field kinds for rb_tree_sample_device -------------------------------------------------- */
#define RB_FIELD_BUMP_POTENTIAL 0 /* k = kb (1 + 0.3 sum_j a_j exp(-|x-c_j|^2/(2 w^2))) + i delta kb     */
#define RB_FIELD_POINT_SOURCE   1 /* f = exp(-|x-x0|^2/(2 w^2)), g = 0                                 */
#define RB_FIELD_PLANE_WAVE     2 /* f = 0, g = i kb (d.n - 1) exp(i kb d.x) (impedance data of the wave) */

/* ---- flags in rb_geom.flags ----------------------------------------------------------------- */
#define RB_FLAG_SKIP_ROOT_RTR 1   /* do not form the root's own RtR (the solve never reads it)         */
#define RB_FLAG_VERBOSE       2   /* print the reference's progress lines to stdout                   */
#define RB_FLAG_NO_GRAPHS     4   /* launch every kernel directly instead of replaying CUDA graphs     */
#define RB_FLAG_ASYNC_FACTOR 16   /* rb_tree_factor returns once the potential is copied and the
                                     factor is enqueued; the next call that needs the factor
                                     (rb_tree_solve, rb_get_solution, rb_tree_get_rtr,
                                     rb_tree_times, another factor) waits for it and reports its
                                     errors (RB_ERR_NUMERIC).  Host right-hand sides of
                                     rb_tree_solve are then copied while the factor runs, and
                                     rb_tree_solve returns once the solution is complete: the
                                     root's own RtR map, which no solve reads, may still be
                                     computed behind it (rb_tree_get_rtr and the next factor
                                     wait for it).                                              */
#define RB_FLAG_MIXED_INT8_TOP 32 /* RB_PREC_MIXED only: the top two merge levels' GEMMs also run on the
                                     int8 tensor-core engine (~1e-11 of max|A| max|B| k); their
                                     interface inversions stay FP64.  Without it those levels are FP64,
                                     as the mixed-precision configuration prescribes.               */
#define RB_FLAG_MERGE_DS      8   /* interface solve as the reference writes it, inv(D) and inv(S)
                                     (compute_RTR, robin_tree_module.f90:449-470), instead of the
                                     default single inversion of K = nu^2 I - (zeta I - T2_ii)(zeta I -
                                     T1_ii); the default also falls back to inv(D), inv(S) by itself
                                     when |nu| < 0.1 max(1, |zeta|)                                    */

typedef struct rb_tree rb_tree;

/* Problem geometry and options: type(elliptic_operator) (derived_type_module.f90:72-84),
 * type(solve_opts) (derived_type_module.f90:309-320), robin_tree%bndry_params
 * (robin_tree_module.f90:61) and the level count L of robin_tree%factor. */
typedef struct rb_geom {
    int32_t d;                 /* elliptic_operator%d; 2 or 3                                       */
    int32_t L;                 /* tree levels; leaves sit at level L                                */
    double  domain[6];         /* elliptic_operator%domain(1:2,1:3), Fortran column-major:
                                  [x_lo, x_hi, y_lo, y_hi, z_lo, z_hi]                              */
    double  h_tgt;             /* solve_opts%h_tgt                                                  */
    double  kb;                /* solve_opts%kb: FD boundary row is u_n + i*kb*u                    */
    double  bndry_params[8];   /* robin_tree%bndry_params(1:2,1:2), complex, column-major,
                                  interleaved: [re11, im11, re21, im21, re12, im12, re22, im22]     */
    int32_t ordering;          /* solve_opts%ordering; only 1 is defined by the reference           */
    int32_t flags;             /* RB_FLAG_*                                                         */
    int64_t device_budget;     /* bytes of device memory the handle may hold; 0 = no limit          */
} rb_geom;

/* Sizes of a created tree. */
typedef struct rb_info {
    int32_t nleaves;           /* 2^L                                                               */
    int32_t leaf_a, leaf_b;    /* leaf grid (ptbox) in x and y                                      */
    int32_t leaf_n;            /* unknowns per leaf = 2(a+b) + a*b, the length of leaf_solution%u   */
    int32_t leaf_nb;           /* boundary points per leaf = 2(a+b)                                 */
    int32_t root_nb;           /* boundary points of the whole domain (length of one g_faces RHS)   */
    int32_t root_a, root_b;    /* grid of the whole domain in x and y: root_nb = 2(root_a + root_b)  */
    double  h_last[3];         /* robin_tree%opts%h after the factorization (the last leaf's h)     */
    int64_t n_interior;        /* nleaves * a * b: length of one potential or source sample array   */
    int64_t device_bytes;      /* device memory currently held by the handle                        */
    int32_t factored;          /* robin_tree%factored                                               */
    int32_t nrhs;              /* right-hand sides held from the last solve                         */
    int32_t d;                 /* dimension, 2 or 3                                                 */
    int32_t leaf_c, root_c;    /* grid in z of a leaf and of the whole domain (1 in 2D); in 3D
                                  leaf_nb = 2(bc + ac + ab), leaf_n = leaf_nb + abc, root_nb likewise,
                                  n_interior = nleaves * abc                                         */
    int32_t reserved;
} rb_info;

/* Builds the tree (robin_tree_factor's setup and bin_tree, robin_tree_module.f90:114-159):
 * validates domain, dimension and det(bndry_params) >= 1e-3, bisects L times and sizes the leaf
 * grids (get_h, fd_module.f90:1060-1084).  Host work only: device memory is allocated by the
 * first factorization.  With geom->device_budget > 0 a tree whose factorization storage cannot
 * fit the budget is refused here with RB_ERR_OUT_OF_MEMORY. */
int rb_tree_create(const rb_geom* geom, rb_tree** out);

/* Releases the handle and all its device memory. */
int rb_tree_destroy(rb_tree* tree);

/* Message of the last failure on `tree`; with NULL, of the last failed rb_tree_create or
 * rb_leaf_rtr_noalloc on this thread. */
const char* rb_last_error(const rb_tree* tree);

int rb_tree_info(const rb_tree* tree, rb_info* info);

/* Coordinates (x, y, z triples) at which the caller evaluates its callbacks, in the order the
 * corresponding sample arrays must use:
 *  RB_POINTS_POTENTIAL: nleaves*a*b (3D: *c) points, leaves in DFS order (child1 first), each
 *                       leaf's interior cell centres x-fastest, then y, then z; each leaf uses
 *                       its own h, as FD_matrix_row does (fd_module.f90:134-145).
 *  RB_POINTS_SOURCE:    the same points computed with robin_tree%opts%h as it stands after the
 *                       factorization (the last leaf's h), as fd_leaf_solve does
 *                       (fd_module.f90:427-431).
 *  RB_POINTS_BOUNDARY:  root_nb face-local coordinates, faces x1 x2 y1 y2 (z1 z2) in turn: the
 *                       concatenation apply_bc builds at the root (robin_tree_module.f90:
 *                       1186-1237) of fd_make_bndry_vec's points (fd_module.f90:636-651), i.e.
 *                       the face's leaves in leaf order, each leaf's points in the face's own
 *                       order (first tangential index fastest).  2D: x-faces carry (y, 0, 0),
 *                       y-faces (x, 0, 0); 3D: x-faces (y, z, 0), y-faces (x, z, 0), z-faces
 *                       (x, y, 0).  The face a point belongs to follows from its index.
 *  RB_POINTS_SOLUTION:  nleaves*leaf_n points of proc2vec (robin_output_module.f90:258-265).
 * `xyz` holds 3 doubles per point.  Requires the tree to be created (not factored). */
int rb_tree_sample_points(const rb_tree* tree, int which, double* xyz);

/* robin_tree%factor(L, op, opts) (robin_tree_module.f90:96-185) with the potential already
 * sampled: `k_centres` = nleaves*a*b complex values at RB_POINTS_POTENTIAL (host memory).
 * Blocks until the factorization is done; robin_tree%f_time is set from device events.
 * The first factorization of a handle launches its kernels directly; the second captures the
 * (fixed) launch sequence into a CUDA graph that later calls replay (RB_FLAG_NO_GRAPHS turns
 * this off; timing modes 1 and 2 launch directly).  The same holds for the solve, per RHS count. */
int rb_tree_factor(rb_tree* tree, const double* k_centres, int precision);

/* As rb_tree_factor, with `d_k_centres` already in device memory.  Asynchronous on the
 * handle's stream when `sync` is 0. */
int rb_tree_factor_device(rb_tree* tree, const double* d_k_centres, int precision, int sync);

/* robin_tree%solve(rhs) (robin_tree_module.f90:198-233) for `nrhs` right-hand sides at once:
 *  f_centres: nrhs * nleaves*a*b complex, RHS-major, each at RB_POINTS_SOURCE; NULL when every
 *             interior source is zero (e.g. plane waves fed through g): the library zeroes its
 *             source array on the device instead of copying one, and solves as for zeros;
 *  g_faces:   nrhs * root_nb complex, RHS-major, each at RB_POINTS_BOUNDARY.
 * Every call applies its own boundary data (the reference applies boundary data only on the
 * first solve of a process, robin_tree_module.f90:1014-1029).  Blocks until done; sets
 * robin_tree%s_time. */
int rb_tree_solve(rb_tree* tree, int nrhs, const double* f_centres, const double* g_faces);

/* As rb_tree_solve with device arrays; asynchronous on the handle's stream when `sync` is 0. */
int rb_tree_solve_device(rb_tree* tree, int nrhs, const double* d_f_centres,
                         const double* d_g_faces, int sync);

/* get_solution(T, u) (robin_output_module.f90:48-75) for right-hand side `irhs`:
 *  u:     nleaves * leaf_n complex (host), leaves in DFS order, each in lin2fgrid order;
 *  boxes: nleaves * 6 doubles (host, may be NULL), each leaf's box(1:2,1:3) column-major. */
int rb_get_solution(const rb_tree* tree, int irhs, double* u, double* boxes);

/* rb_get_solution without waiting for the copy (beyond the reference, whose get_solution returns
 * filled arrays): enqueues the device -> host copy of right-hand side irhs's solution into u on a
 * stream of its own, behind the solve that wrote it, and returns; boxes (may be NULL) are filled
 * at once.  u must stay valid and untouched until rb_tree_sync(tree) returns; with pinned host
 * memory the copy runs beside later work, e.g. the next factorization.  A later solve waits on the
 * device for these copies before it overwrites the solution. */
int rb_get_solution_async(const rb_tree* tree, int irhs, double* u, double* boxes);
/* Waits until every copy rb_get_solution_async enqueued for this handle has landed. */
int rb_tree_sync(const rb_tree* tree);

/* All right-hand sides' solutions into device memory: nrhs * nleaves * leaf_n complex,
 * RHS-major.  Asynchronous on the handle's stream when `sync` is 0. */
int rb_get_solution_device(const rb_tree* tree, double* d_u, int sync);

/* robin_tree%f_time and robin_tree%s_time in seconds (device-event timing). */
int rb_tree_times(const rb_tree* tree, double* f_time, double* s_time);

/* The handle's CUDA stream (a cudaStream_t), for callers that order their own work with it. */
void* rb_tree_stream(const rb_tree* tree);

/* Device-event timing.  mode 0: off.  mode 1: per stage (leaf stage, each merge level, forward,
 * backward, leaf recovery) of the last factor and solve.  mode 2: one entry per kernel launch
 * (a whole Gauss-Jordan batch counts as one), accumulated over calls until
 * rb_tree_clear_stage_times, with each entry's algorithmic flop count (8mnk for a complex GEMM,
 * 8m^3 per Gauss-Jordan inverse, 0 for data-movement kernels).  rb_tree_stage_times writes
 * min(n, count) entries (any output pointer may be NULL) and returns the count; names point to
 * strings owned by the handle.  Entries are complete after the handle's stream is synchronized. */
int rb_tree_set_timing(rb_tree* tree, int mode);
int rb_tree_stage_times(const rb_tree* tree, double* ms, double* flops, const char** names, int n);
int rb_tree_clear_stage_times(rb_tree* tree);

/* Shape of level `level` (0 = root, L = leaves) into shape[0..3]: the node count and the grid
 * (ptbox) of each node in x, y and z (robin_tree_module.f90:404-407 for merged nodes; z = 1 in
 * 2D).  `shape` holds 4 entries. */
int rb_tree_level_shape(const rb_tree* tree, int level, int32_t* shape);

/* Robin-to-Robin matrix of node `node` (0-based, left to right; leaves in DFS order) of level
 * `level` (0 = root, L = leaves) after the factorization, into `out`: nb x nb complex,
 * column-major, rows/columns in face order x1 x2 y1 y2 -- the blocks node%RtR(row,col)
 * (robin_tree_module.f90:782-793 for leaves, :538-615 for merges) assembled into one matrix.
 * RB_ERR_INVALID for the root when RB_FLAG_SKIP_ROOT_RTR is set. */
int rb_tree_get_rtr(const rb_tree* tree, int level, int node, double* out);

/* ---- beyond the reference's factor/solve: device-side inputs, error reports, persistence ---- */

/* Samples a standard potential or right-hand-side family on the device, at exactly the points
 * rb_tree_sample_points lists, so that the inputs of rb_tree_factor_device / rb_tree_solve_device
 * never cross PCIe (the reference evaluates its callbacks point by point on the host,
 * fd_module.f90:136-145, 427-431, 636-651).  Formulas and the rounding of their exponents
 * follow the synthetic problems' host definitions; exp, sin and cos are CUDA's.
 *  RB_FIELD_BUMP_POTENTIAL: params = kb, delta, w, then (cx, cy, a) for each of `count` bumps;
 *                           writes n_interior values to d_f (d_g unused).
 *  RB_FIELD_POINT_SOURCE:   params = (x0, y0, w) per right-hand side, `count` of them; writes
 *                           count * n_interior f values to d_f and zeros to d_g (either may be NULL).
 *  RB_FIELD_PLANE_WAVE:     params = (kb, dx, dy) per right-hand side (unit direction d); writes
 *                           count * root_nb g values to d_g and zeros to d_f (either may be NULL).
 * Runs on the handle's stream; asynchronous when `sync` is 0.  Needs only rb_tree_create. */
int rb_tree_sample_device(rb_tree* tree, int kind, int count, const double* params, double* d_f,
                          double* d_g, int sync);

/* check_solution (robin_output_module.f90:84-134) on the device: per leaf, the norm of
 * u - u_exact (rel = 0) or of (u - u_exact) / u_exact (rel = 1) for right-hand side `irhs` of
 * the last solve, norm 1 (sum), 2 (Euclidean) or anything else (maximum) of the moduli.
 * u_exact: nleaves * leaf_n complex at RB_POINTS_SOLUTION (host memory; _device: device memory).
 * err: nleaves doubles (host).  The solution itself stays on the device. */
int rb_check_solution(const rb_tree* tree, int irhs, const double* u_exact, int norm, int rel, double* err);
int rb_check_solution_device(const rb_tree* tree, int irhs, const double* d_u_exact, int norm, int rel,
                             double* err);

/* Writes the factorized tree (its rb_geom and every array the solve reads: leaf factors, level
 * RtR maps, interface inverses and the levels' [Y1; Y2]) to `path`, and rebuilds a handle from
 * such a file, ready to solve, without factoring again.  No counterpart in the reference (its write_variable is a
 * stub, robin_output_module.f90:157-221).  The file holds raw complex128 arrays of this
 * library's layout; rb_tree_load refuses files of another version, tree or interface form. */
int rb_tree_save(const rb_tree* tree, const char* path);
int rb_tree_load(const char* path, rb_tree** out);

/* Iterative refinement of solves against a RB_PREC_MIXED factorization.  The reference solves
 * with its one FP64 factorization (robin_tree_solve, robin_tree_module.f90:198-233) and has no
 * counterpart; this is the `tol` of a mixed-precision solve.  Each solve applies corrections
 * d = M^-1 (b - A x), with the global FD system's residual b - A x in FP64, until every right-hand
 * side's estimated relative max-norm error rho |d| / |x| (rho the observed contraction factor) is
 * below tol / 10, or fails with RB_ERR_NUMERIC after max_iter corrections or when the iteration
 * does not contract.  Defaults: tol = 1e-10, max_iter = 8.  Solves of an FP64 factorization are
 * direct and ignore these settings. */
int rb_tree_set_refinement(rb_tree* tree, double tol, int max_iter);

/* The last mixed-precision solve: corrections applied, the largest contraction factor seen, the
 * estimated relative error of the returned solutions and the last residual max |b - A x| / max |x|
 * (any output pointer may be NULL). */
int rb_tree_refine_info(const rb_tree* tree, int32_t* iters, double* contraction, double* est_err,
                        double* residual);

/* Number of this library's kernels launched by the last factor and the last solve. */
int rb_tree_launch_counts(const rb_tree* tree, int64_t* factor_launches, int64_t* solve_launches);

/* ---- forests: many trees factored in one level-synchronous schedule ---------------------------
 *
 * No counterpart in the reference, which factors one tree by a serial recursion (compute_RTR,
 * robin_tree_module.f90:375-401).  A forest references existing trees (created with
 * rb_tree_create, any sizes, single-inversion K-form merges; still owned by the caller) and factors
 * them together: aligned by height above their leaves, every merge stage of a height runs as ONE
 * launch over the concatenated descriptors of all trees (uneven interface lengths in one launch),
 * with one Gauss-Jordan launch per distinct interface size; the schedule is captured into a CUDA
 * graph and replayed.  A project autotuner (autotune != 0 on a factor call) times each applicable
 * FP64 GEMM tile shape on every concatenated stage once, keeps the fastest, and caches the choices
 * for the process by stage shape.  After rb_forest_factor every tree is factored (FP64) and is
 * solved with rb_tree_solve as usual. */
typedef struct rb_forest rb_forest;
int rb_forest_create(rb_tree* const* trees, int ntrees, rb_forest** out);
int rb_forest_destroy(rb_forest* forest);
const char* rb_forest_last_error(const rb_forest* forest);
/* d_k[i]: device array of tree i's potential samples (n_interior complex at RB_POINTS_POTENTIAL).
 * Blocks until the factorizations are done; sets every tree's f_time to the forest's time. */
int rb_forest_factor(rb_forest* forest, const double* const* d_k, int autotune);
/* Device time of the last forest factor, the launches of its schedule, and the stages whose tile
 * shape the autotuner fixed (any output pointer may be NULL). */
int rb_forest_info(const rb_forest* forest, double* f_time, int64_t* launches, int32_t* tuned_stages);
/* The autotuner's measurements: min(n, count) entries of (height, stage 0..4 = K, B1, Y1, Y2, parent
 * map, engine id, ms per launch; -1 for a shape that could not launch on that stage); returns the
 * count.  rb_gemm_engine_name names an engine id. */
int rb_forest_tuning(const rb_forest* forest, int32_t* height, int32_t* stage, int32_t* engine, double* ms, int n);
const char* rb_gemm_engine_name(int engine);

/* ---- serving: resident factorized trees and a continuously batched request loop ---------------
 *
 * No counterpart in the reference, which factors one tree and solves one right-hand side per call,
 * once per process (robin_tree_solve, robin_tree_module.f90:198-233, 1014-1029).  A server owns
 * several trees on the current device.  Each tree has a worker thread and its own CUDA streams, so
 * the trees' work overlaps on the device.  Solve requests queued for a tree are merged, up to
 * max_batch_rhs right-hand sides, into one batched sweep when the tree's previous work is done;
 * requests arriving meanwhile form the next batch.  A factor request is ordered with its tree's
 * solves: solves submitted before it use the old factorization.  A tree's first factorization
 * reserves its estimated device footprint (factor storage, buffers of a full batch, input staging)
 * against the server's budget and waits while other trees' reservations leave too little room.
 * Latency is measured from the request's arrival stamp (server clock, rb_server_now; a negative
 * stamp means the submit time) to its completion with the solution in host memory. */
typedef struct rb_server rb_server;

typedef struct rb_server_opts {
    int64_t device_budget;     /* bytes the trees and their buffers may reserve together;
                                  0 = 90% of the device memory free at creation                     */
    int32_t max_batch_rhs;     /* most right-hand sides merged into one sweep (0: 64)               */
    int32_t precision;         /* RB_PREC_FP64 or RB_PREC_MIXED for every factorization             */
    double  tol;               /* refinement tolerance of mixed-precision solves (0: 1e-10)         */
} rb_server_opts;

typedef struct rb_server_stats {
    int64_t solves, rhs, factors, batches, failed;   /* completed requests since the last reset    */
    double  p50_ms, p99_ms, mean_ms, max_ms;         /* solve latency: arrival -> solution on host */
    double  factor_p50_ms, factor_max_ms;            /* factor latency: arrival -> factor resident */
    int64_t reserved_bytes;                          /* device memory reserved by the trees        */
} rb_server_stats;

int rb_server_create(const rb_server_opts* opts, rb_server** out);
/* Stops the workers (queued requests fail), releases every tree and buffer. */
int rb_server_destroy(rb_server* server);
const char* rb_server_last_error(const rb_server* server);
/* Seconds since the server was created: the clock of arrival stamps and latencies. */
double rb_server_now(const rb_server* server);
/* Registers a tree geometry (as rb_tree_create; rb_geom.device_budget and RB_FLAG_ASYNC_FACTOR
 * are ignored) and starts its worker; device memory is reserved by its first factorization. */
int rb_server_add_tree(rb_server* server, const rb_geom* geom, int32_t* tree_id);
int rb_server_tree_info(rb_server* server, int32_t tree_id, rb_info* info);
/* Factor request: host potential samples k (n_interior complex at RB_POINTS_POTENTIAL, copied
 * before returning), or k = NULL and the RB_FIELD_BUMP_POTENTIAL parameters (kb, delta, w, then
 * (cx, cy, a) per bump, field_count bumps; copied) sampled on the device. */
int rb_server_submit_factor(rb_server* server, int32_t tree_id, const double* k, int field_count,
                            const double* field_params, double arrival, int64_t* request);
/* Solve request of nrhs <= max_batch_rhs right-hand sides: field = RB_FIELD_POINT_SOURCE or
 * RB_FIELD_PLANE_WAVE with 3 parameters per right-hand side (as rb_tree_sample_device; copied),
 * or field = -1 and host arrays f (nrhs * n_interior complex) and g (nrhs * root_nb complex), which
 * must stay valid until the request completes (NULL = zero).  u: host buffer of
 * nrhs * nleaves * leaf_n complex that receives the solutions (NULL: not copied out). */
int rb_server_submit_solve(rb_server* server, int32_t tree_id, int nrhs, int field, const double* params,
                           const double* f, const double* g, double* u, double arrival, int64_t* request);
/* Waits for a request (timeout_s < 0: without limit).  Returns its status (RB_OK or RB_ERR_*, with
 * the message in rb_server_last_error) and forgets it, or 1 if it is still pending at the timeout. */
int rb_server_wait(rb_server* server, int64_t request, double timeout_s);
/* Counters and latency percentiles of the requests completed since the last reset (reset != 0
 * clears them after reading). */
int rb_server_get_stats(rb_server* server, rb_server_stats* stats, int reset);

/* Leaf Robin-to-Robin maps for callers that cannot allocate device memory.  No counterpart in
 * the reference (whose leaf RtR is node%RtR after RTR_solve, robin_tree_module.f90:728-799; the
 * maps this writes are those of rb_tree_factor's leaves, see rb_tree_get_rtr).
 *
 * Meant for callers that must not call cudaMalloc: a framework that owns the device's memory
 * through its own pool (or has reserved it up front) and forbids allocations by libraries, or
 * a latency-critical loop where cudaMalloc's implicit device synchronisation is unacceptable.
 * This entry point allocates nothing and calls no allocating routine; its working memory is a
 * file-scope device array of 32 MiB that every GPU holds from the library's load until exit.
 *
 *  a, b      leaf grid (ptbox) in x and y, each >= 3
 *  kb        solve_opts%kb
 *  d_h       device, 2*nleaves doubles: each leaf's (hx, hy)
 *  d_k       device, nleaves*a*b complex: each leaf's potential at its interior cell centres
 *            (x fastest), as rb_tree_factor's samples for one leaf
 *  d_rtr     device, nleaves*nb*nb complex (nb = 2(a+b)) output: each leaf's RtR, column-major,
 *            faces x1 x2 y1 y2 -- what rb_tree_get_rtr(tree, L, i) returns for a factored tree
 *  stream    cudaStream_t to run on (NULL = the default stream); the call returns after the
 *            stream's work is done
 * Limit: nleaves * (b*a^2 + nb*(nb + a*b)) * 16 + 256 bytes of scratch must fit 32 MiB (85 leaves
 * of 16x16); larger batches are refused with RB_ERR_INVALID and a message giving the limit.
 * The first call on a device looks up the array's address (cudaGetSymbolAddress) with that device
 * current; make that first call before starting any stream capture.  All calls share the array
 * and it keeps the previous call's contents: calls whose GPU work overlaps (several streams or
 * host threads on one device) race on it.  Errors: RB_ERR_INVALID, RB_ERR_CUDA, RB_ERR_NUMERIC
 * (zero pivot); the message is rb_last_error(NULL). */
int rb_leaf_rtr_noalloc(int a, int b, double kb, const double* d_h, const double* d_k, int nleaves,
                        double* d_rtr, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ROBIN_B200_H */
