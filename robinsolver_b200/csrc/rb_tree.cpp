// rb_tree.cpp -- the C-ABI of the B200 HPS factor/solve (include/robin_b200.h).
//
// Host runtime: builds the tree plan (no device work), owns the device memory of a tree, builds
// the GEMM / Gauss-Jordan descriptor batches once per tree (factor) and once per right-hand-side
// count (solve), and launches the level-by-level stages on the handle's stream.
//
// Factor (robin_tree_factor -> compute_RTR, robin_tree_module.f90:96-185, 375-650):
//   leaves:  block-tridiagonal factor of S = A_ii - A_ib A_bb^-1 A_bi from the potential
//            samples and Y = R A^-1 (RtR in its first nb columns), one CTA per leaf (rb_leaf.cu)
//   level l = L-1 .. 0, all nodes of the level in one launch per stage.  [Y1; Y2] =
//   M^-1 blockdiag(T1_iN, T2_iN) solves the interface system M = [[A1, nu I], [nu I, A2]],
//   A1 = zeta I - T1_ii, A2 = zeta I - T2_ii, then
//            parent RtR = T_NN + [T1_Ni Y1; T2_Ni Y2], scattered into the parent's face order
//   (Y1 = [C11, -C12] and Y2 = [-C21, C22] in the reference's names, :482-615).  Two forms:
//   K form (default): one inversion per node, K = nu^2 I - A2 A1 (for the impedance pair zeta = 0,
//            nu = -1 this is the familiar I - T2_ii T1_ii), Y1 = inv(K) [-A2 T1_iN, nu T2_iN],
//            Y2 = ([T1_iN, 0] - A1 Y1) / nu;
//   D/S form (the reference's, RB_FLAG_MERGE_DS, or |nu| small against |zeta|):
//            inv(D), D = A2;  inv(S), S = A1 - nu^2 inv(D);  Y2R = inv(D) T2_iN;
//            Y1 = inv(S) [T1_iN, -nu Y2R];  Y2 = [0, Y2R] - nu inv(D) Y1.
// Solve (forward_sub / backward_sub, robin_tree_module.f90:813-1146), all RHS at once:
//   forward:  leaf h = Y(:, nb:) f;  per level (g1_i, g2_i) = M^-1 (h1_i, h2_i) and the parent's
//             h = h_N + T_Ni g_i
//   root:     its forward and backward steps are one, g_i = M^-1 (h_i + T_iN g_N) with g_N the
//             boundary data; x = h + T_iN g_N (and in the K form nu x2 - A2 x1) runs before the
//             root's inverse is ready
//   backward: per level below the root, the children's g_N from the parent and
//             g_i += M^-1 T_iN g_N = [Y1; Y2] g_N with the level's stored Y (one GEMM per level
//             instead of four dependent ones); leaf u = A^-1 [g; f] through the leaf's block factors.
//   M^-1 (x1, x2), K form: y1 = inv(K)(nu x2 - A2 x1), y2 = (x1 - A1 y1) / nu;  D/S form:
//   w = inv(D) x2; y1 = inv(S)(x1 - nu w); y2 = w - nu inv(D) y1 (apply_invm, :1252).
#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <functional>
#include <map>
#include <vector>

#include "robin_b200.h"
#include "rb_kernels.h"
#include "rb_plan.hpp"
#include "rb_tree_impl.hpp"

namespace rb {
static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
static void g_launches_add(long long d) { g_launches.fetch_add(d, std::memory_order_relaxed); }
}  // namespace rb

static thread_local std::string g_create_error;

namespace rb {
void set_thread_error(const char* msg) { g_create_error = msg ? msg : ""; }
}  // namespace rb

using namespace rb;


// ---------------------------------------------------------------------------------------------------
#define RB_CK(call)                                                                              \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            t->err = std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call;        \
            return RB_ERR_CUDA;                                                                  \
        }                                                                                        \
    } while (0)

static int fail(rb_tree* t, int code, const std::string& msg) {
    t->err = msg;
    return code;
}

static int dev_alloc(rb_tree* t, std::vector<DevBuf>& list, size_t bytes, void** out) {
    *out = nullptr;
    if (bytes == 0) return RB_OK;
    bytes = (bytes + 255) & ~size_t(255);
    if (t->budget > 0 && t->held + (int64_t)bytes > t->budget)
        return fail(t, RB_ERR_OUT_OF_MEMORY, "device budget exceeded: need " + std::to_string(t->held + bytes) +
                                                 " bytes, budget " + std::to_string(t->budget));
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(t, e == cudaErrorMemoryAllocation ? RB_ERR_OUT_OF_MEMORY : RB_ERR_CUDA,
                    std::string("cudaMalloc of ") + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
    }
    list.push_back({p, bytes});
    t->held += (int64_t)bytes;
    *out = p;
    return RB_OK;
}

template <class T>
static int alloc_n(rb_tree* t, std::vector<DevBuf>& list, size_t n, T** out) {
    void* p = nullptr;
    int rc = dev_alloc(t, list, n * sizeof(T), &p);
    *out = static_cast<T*>(p);
    return rc;
}

static void free_list(rb_tree* t, std::vector<DevBuf>& list) {
    for (auto& b : list) {
        cudaFree(b.p);
        t->held -= (int64_t)b.bytes;
    }
    list.clear();
}

static int upload_gemm(rb_tree* t, std::vector<DevBuf>& list, const std::vector<GemmDesc>& h, GemmBatch& b) {
    b = GemmBatch();
    b.count = (int)h.size();
    if (h.empty()) return RB_OK;
    int rc = alloc_n(t, list, h.size(), &b.d_desc);
    if (rc) return rc;
    RB_CK(cudaMemcpy(b.d_desc, h.data(), h.size() * sizeof(GemmDesc), cudaMemcpyHostToDevice));
    b.kcontig = true;
    for (const auto& d : h) {
        b.max_m = std::max(b.max_m, d.m);
        b.max_n = std::max(b.max_n, d.n);
        b.max_k = std::max(b.max_k, d.k);
        b.flops += 8.0 * d.m * d.n * d.k;
        b.kcontig = b.kcontig && gemm_k_contiguous(d);
    }
    return RB_OK;
}

static int upload_gj(rb_tree* t, std::vector<DevBuf>& list, const std::vector<GJDesc>& h, int m, GJBatch& b) {
    b = GJBatch();
    b.count = (int)h.size();
    b.m = m;
    if (h.empty()) return RB_OK;
    int rc = alloc_n(t, list, h.size(), &b.d_desc);
    if (rc) return rc;
    RB_CK(cudaMemcpy(b.d_desc, h.data(), h.size() * sizeof(GJDesc), cudaMemcpyHostToDevice));
    return RB_OK;
}

static ZView band_view(const z* p, long long ld, int rs, int rl, int cs, int cl) {
    ZView v = zview(p, ld);
    v.rs = rs; v.rl = rl; v.cs = cs; v.cl = cl;
    return v;
}

static GemmDesc gdesc(int m, int n, int k, ZView A, ZView B, ZOut D, z alpha) {
    GemmDesc g;
    std::memset(&g, 0, sizeof(g));
    g.A = A; g.B = B; g.C = zview(nullptr, 1); g.D = D;
    g.alpha = alpha; g.beta = zmk(0.0, 0.0);
    g.m = m; g.n = n; g.k = k;
    return g;
}

static ChildStore child_store(const rb_tree* t, int l) {   // storage of level l+1's RtR
    const Plan& P = t->P;
    ChildStore c;
    if (l + 1 == P.L) {
        c.rtr = t->leaf_Y;
        c.stride = (long long)P.leaf_nb() * P.leaf_n();
        c.ld = P.leaf_nb();
    } else {
        const int nbc = P.lv[l + 1].nb;
        c.rtr = t->rtr[l + 1];
        c.stride = (long long)nbc * nbc;
        c.ld = nbc;
    }
    return c;
}

// ---------------------------------------------------------------------------------------------------
static int timer_open(rb_tree* t, const char* name, double flops) {
    if (t->ev_used + 2 > (int)t->ev_pool.size()) {
        for (int i = 0; i < 64; ++i) {
            cudaEvent_t e;
            RB_CK(cudaEventCreate(&e));
            t->ev_pool.push_back(e);
        }
    }
    StageTimer st{name, flops, t->ev_used};
    t->ev_used += 2;
    RB_CK(cudaEventRecord(t->ev_pool[st.ev], t->stream));
    t->timers.push_back(st);
    return RB_OK;
}
static int timer_close(rb_tree* t) {
    RB_CK(cudaEventRecord(t->ev_pool[t->timers.back().ev + 1], t->stream));
    return RB_OK;
}
// stage granularity (timing == 1)
static int timer_begin(rb_tree* t, const char* name) { return t->timing == 1 ? timer_open(t, name, 0.0) : RB_OK; }
static int timer_end(rb_tree* t) { return t->timing == 1 ? timer_close(t) : RB_OK; }
// launch granularity (timing == 2): one entry per kernel launch (or per Gauss-Jordan batch)
static int ltimer_begin(rb_tree* t, const char* name, double flops) {
    return t->timing == 2 ? timer_open(t, name, flops) : RB_OK;
}
static int ltimer_end(rb_tree* t) { return t->timing == 2 ? timer_close(t) : RB_OK; }
static void timers_collect(rb_tree* t) {
    for (auto& st : t->timers) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, t->ev_pool[st.ev], t->ev_pool[st.ev + 1]) == cudaSuccess)
            t->stage_ms.push_back({st.name, (double)ms, st.flops});
    }
    t->timers.clear();
    t->ev_used = 0;
}

static void drop_graph(cudaGraphExec_t& g) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
}

// runs `body` directly, or captures it once into `gx` and replays it; `launches` receives the
// number of kernels the sequence launches
template <class F>
static int run_graphed(rb_tree* t, cudaGraphExec_t& gx, long long& gx_launches, int& runs, F body) {
    if (!t->graphs || t->timing != 0 || runs == 0) {
        ++runs;
        return body();
    }
    if (!gx) {
        const long long l0 = launch_count();
        RB_CK(cudaStreamBeginCapture(t->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = body();
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(t->stream, &g);
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            if (rc) return rc;
            t->err = std::string("CUDA graph capture failed: ") + cudaGetErrorString(e);
            return RB_ERR_CUDA;
        }
        const cudaError_t ei = cudaGraphInstantiate(&gx, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            gx = nullptr;
            t->err = std::string("CUDA graph instantiation failed: ") + cudaGetErrorString(ei);
            return RB_ERR_CUDA;
        }
        gx_launches = launch_count() - l0;
        g_launches_add(-gx_launches);      // captured, not yet launched
    }
    RB_CK(cudaGraphLaunch(gx, t->stream));
    g_launches_add(gx_launches);
    ++runs;
    return RB_OK;
}

// ---------------------------------------------------------------------------------------------------
static int ensure_factor_storage(rb_tree* t) {
    if (t->factor_ready) return RB_OK;
    const Plan& P = t->P;
    const int L = P.L, nl = P.nleaves(), a = P.leaf_a(), b = P.leaf_b(), nint = P.leaf_interior();
    const int nb = P.leaf_nb(), n = P.leaf_n();
    int rc;
    RB_CK(cudaGetDevice(&t->device));
    if (!t->stream) RB_CK(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking));
    {
        // the level chain (stream2) and B1 (stream4) above the main stream, so that their CTAs are
        // dispatched ahead of the waves of the large GEMM they overlap; the solve (stream3) above
        // both
        int least = 0, greatest = 0;
        RB_CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        const int side = greatest < least ? std::max(greatest, least - 1 - (least - greatest) / 2) : least;
        if (!t->stream2) RB_CK(cudaStreamCreateWithPriority(&t->stream2, cudaStreamNonBlocking, side));
        if (!t->stream4) RB_CK(cudaStreamCreateWithPriority(&t->stream4, cudaStreamNonBlocking, side));
    }
    if (!t->stream3) {
        // the solve runs here beside a factor: at the highest priority its small, latency-bound
        // kernels take SMs ahead of the factor's large GEMMs as their CTAs retire
        int least = 0, greatest = 0;
        RB_CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        RB_CK(cudaStreamCreateWithPriority(&t->stream3, cudaStreamNonBlocking, greatest));
    }
    if (!t->ev_copy) RB_CK(cudaEventCreateWithFlags(&t->ev_copy, cudaEventDisableTiming));
    for (auto& e : t->ev)
        if (!e) RB_CK(cudaEventCreate(&e));
    if (!t->h_status) {
        RB_CK(cudaMallocHost(&t->h_status, 2 * sizeof(int)));
        t->h_status[0] = t->h_status[1] = 0;
    }
    t->ev_fork.assign(L, nullptr);
    t->ev_join.assign(L, nullptr);
    t->ev_lvl.assign(L + 1, nullptr);
    for (int l = 0; l <= L; ++l) RB_CK(cudaEventCreateWithFlags(&t->ev_lvl[l], cudaEventDisableTiming));
    if (!t->ev_root_forms) RB_CK(cudaEventCreateWithFlags(&t->ev_root_forms, cudaEventDisableTiming));
    if (!t->ev_root_gj) RB_CK(cudaEventCreateWithFlags(&t->ev_root_gj, cudaEventDisableTiming));
    for (auto* v : {&t->ev_face, &t->ev_rest, &t->ev_d, &t->ev_m1, &t->ev_m3}) {
        v->assign(L + 1, nullptr);
        for (auto& e : *v) RB_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    for (int l = 0; l < L; ++l) {
        RB_CK(cudaEventCreateWithFlags(&t->ev_fork[l], cudaEventDisableTiming));
        RB_CK(cudaEventCreateWithFlags(&t->ev_join[l], cudaEventDisableTiming));
    }
    if ((rc = alloc_n(t, t->bufs, (size_t)P.d * nl, &t->d_h))) return rc;
    RB_CK(cudaMemcpy(t->d_h, P.leaf_h.data(), (size_t)P.d * nl * sizeof(double), cudaMemcpyHostToDevice));
    if ((rc = alloc_n(t, t->bufs, (size_t)nl * nint, &t->d_k))) return rc;
    if (P.d == 2) {
        if ((rc = alloc_n(t, t->bufs, (size_t)nl * b * a * a, &t->leaf_sinv))) return rc;
    } else {
        // 3D: each leaf's dense FD matrix, inverted in place by the batched Gauss-Jordan kernels
        if (n > 1024) return fail(t, RB_ERR_UNSUPPORTED, "3D leaf larger than 1024 unknowns");
        if ((rc = alloc_n(t, t->bufs, (size_t)nl * n * n, &t->leaf_sinv))) return rc;
        if ((rc = alloc_n(t, t->bufs, (size_t)nl * n, &t->leaf_ipiv))) return rc;
        const long long ws = gj_workspace_elems(n);
        if ((rc = alloc_n(t, t->bufs, (size_t)std::max<long long>(1, nl * ws), &t->leaf_gjwork))) return rc;
        std::vector<GJDesc> v(nl);
        for (int i = 0; i < nl; ++i) {
            v[i].A = t->leaf_sinv + (long long)i * n * n;
            v[i].ld = n;
            v[i].ipiv = t->leaf_ipiv + (long long)i * n;
            v[i].Zb = t->leaf_gjwork + (long long)i * ws;
        }
        if ((rc = upload_gj(t, t->bufs, v, n, t->gj_leaf))) return rc;
    }
    if ((rc = alloc_n(t, t->bufs, (size_t)nl * nb * n, &t->leaf_Y))) return rc;
    if ((rc = alloc_n(t, t->bufs, 1, &t->d_status))) return rc;
    t->rtr.assign(L, nullptr);
    t->dinv.assign(L, nullptr);
    t->sinv.assign(L, nullptr);
    t->kinv.assign(L, nullptr);
    t->d_pmap1.assign(L, nullptr);
    t->d_pmap2.assign(L, nullptr);
    t->d_pmapc.assign(L, nullptr);
    t->Y1.assign(L, nullptr);
    t->Y2.assign(L, nullptr);
    for (int l = 0; l < L; ++l) {
        const PlanLevel& p = P.lv[l];
        if (!(l == 0 && t->skip_root))
            if ((rc = alloc_n(t, t->bufs, (size_t)p.nnodes * p.nb * p.nb, &t->rtr[l]))) return rc;
        if ((rc = alloc_n(t, t->bufs, (size_t)p.nnodes * p.m * p.m, &t->dinv[l]))) return rc;
        if ((rc = alloc_n(t, t->bufs, (size_t)p.nnodes * p.m * p.m, &t->sinv[l]))) return rc;
        if (t->kform)
            if ((rc = alloc_n(t, t->bufs, (size_t)p.nnodes * p.m * p.m, &t->kinv[l]))) return rc;
        if ((rc = alloc_n(t, t->bufs, p.pmap1.size(), &t->d_pmap1[l]))) return rc;
        if ((rc = alloc_n(t, t->bufs, p.pmap2.size(), &t->d_pmap2[l]))) return rc;
        RB_CK(cudaMemcpy(t->d_pmap1[l], p.pmap1.data(), p.pmap1.size() * sizeof(int), cudaMemcpyHostToDevice));
        RB_CK(cudaMemcpy(t->d_pmap2[l], p.pmap2.data(), p.pmap2.size() * sizeof(int), cudaMemcpyHostToDevice));
        std::vector<int> pc(p.pmap1);
        pc.insert(pc.end(), p.pmap2.begin(), p.pmap2.end());
        if ((rc = alloc_n(t, t->bufs, pc.size(), &t->d_pmapc[l]))) return rc;
        RB_CK(cudaMemcpy(t->d_pmapc[l], pc.data(), pc.size() * sizeof(int), cudaMemcpyHostToDevice));
        const size_t ny = (size_t)p.nnodes * p.m * (p.n1 + p.n2);
        if ((rc = alloc_n(t, t->bufs, ny, &t->Y1[l]))) return rc;
        if ((rc = alloc_n(t, t->bufs, ny, &t->Y2[l]))) return rc;
    }
    // Gauss-Jordan workspace: the largest batch of one level's nodes
    size_t wmax = 1, imax = 1;
    for (int l = 0; l < L; ++l) {
        const PlanLevel& p = P.lv[l];
        wmax = std::max(wmax, (size_t)p.nnodes * (size_t)gj_workspace_elems(p.m));
        imax = std::max(imax, (size_t)p.nnodes * p.m);
    }
    if ((rc = alloc_n(t, t->bufs, std::max<size_t>(wmax, 1), &t->gj_work))) return rc;
    if ((rc = alloc_n(t, t->bufs, imax, &t->gj_ipiv))) return rc;

    auto gj_descs = [&](z* base, long long stride, int ld, int count, int m) {
        std::vector<GJDesc> v(count);
        const long long ws = gj_workspace_elems(m);
        for (int i = 0; i < count; ++i) {
            v[i].A = base + (long long)i * stride;
            v[i].ld = ld;
            v[i].ipiv = t->gj_ipiv + (long long)i * m;
            v[i].Zb = t->gj_work + (long long)i * ws;
        }
        return v;
    };
    t->gj_d.resize(L);
    t->gj_s.resize(L);
    t->gj_k.resize(L);
    t->fK.resize(L); t->fM1.resize(L); t->fM2.resize(L); t->fM3.resize(L); t->fM4.resize(L);
    t->fM4F.assign(L, GemmBatch()); t->fM4N.assign(L, GemmBatch());
    const z one = zmk(1.0, 0.0);
    const z mone = zmk(-1.0, 0.0);
    const z mnu = zneg(t->nu);
    const z rnu = zrcp(t->nu), mrnu = zneg(rnu);
    for (int l = 0; l < L; ++l) {
        const PlanLevel& p = P.lv[l];
        const int m = p.m, n1 = p.n1, n2 = p.n2, o1 = p.o1, o2 = p.o2, nn = p.nnodes;
        if (t->kform) {
            if ((rc = upload_gj(t, t->bufs, gj_descs(t->kinv[l], (long long)m * m, m, nn, m), m, t->gj_k[l]))) return rc;
        } else {
            if ((rc = upload_gj(t, t->bufs, gj_descs(t->dinv[l], (long long)m * m, m, nn, m), m, t->gj_d[l]))) return rc;
            if ((rc = upload_gj(t, t->bufs, gj_descs(t->sinv[l], (long long)m * m, m, nn, m), m, t->gj_s[l]))) return rc;
        }
        const ChildStore cs = child_store(t, l);
        std::vector<GemmDesc> mk, m1, m2, m3, m4, m4f, m4n;
        // The pipelined factor's row split of this level's parent maps (levels 1..L-1, K form): for
        // a node that is its parent's child1 (par 0) or child2 (par 1), the rows of its map on the
        // face the parent merges across, and the others.  Per child a of the node: sel = the rows'
        // physical rows in child a's map (its non-interface points t, past the interface band),
        // out = their rows in the node's map (pmap_a[t]).
        int* d_sel[2][2][2] = {};
        int* d_out[2][2][2] = {};
        int cnt[2][2][2] = {};
        const bool split = l >= 1 && t->kform;
        if (split) {
            const PlanLevel& pp = P.lv[l - 1];
            for (int par = 0; par < 2; ++par) {
                const int f = par == 0 ? pp.iface1 : pp.iface2;
                const int lo = p.off[f - 1], hi = lo + p.pf[f - 1];
                for (int a = 0; a < 2; ++a) {
                    const std::vector<int>& pm = a == 0 ? p.pmap1 : p.pmap2;
                    const int oa = a == 0 ? o1 : o2;
                    std::vector<int> sel[2], out[2];
                    for (int tt = 0; tt < (int)pm.size(); ++tt) {
                        const int kind = (pm[tt] >= lo && pm[tt] < hi) ? 0 : 1;
                        sel[kind].push_back(tt < oa ? tt : tt + m);
                        out[kind].push_back(pm[tt]);
                    }
                    for (int kind = 0; kind < 2; ++kind) {
                        cnt[par][a][kind] = (int)sel[kind].size();
                        if (sel[kind].empty()) continue;
                        if ((rc = alloc_n(t, t->bufs, sel[kind].size(), &d_sel[par][a][kind]))) return rc;
                        if ((rc = alloc_n(t, t->bufs, out[kind].size(), &d_out[par][a][kind]))) return rc;
                        RB_CK(cudaMemcpy(d_sel[par][a][kind], sel[kind].data(), sel[kind].size() * sizeof(int),
                                         cudaMemcpyHostToDevice));
                        RB_CK(cudaMemcpy(d_out[par][a][kind], out[kind].data(), out[kind].size() * sizeof(int),
                                         cudaMemcpyHostToDevice));
                    }
                }
            }
        }
        for (int i = 0; i < nn; ++i) {
            const z* r1 = cs.rtr + (2LL * i) * cs.stride;
            const z* r2 = cs.rtr + (2LL * i + 1) * cs.stride;
            const long long ld = cs.ld;
            z* dv = t->dinv[l] + (long long)i * m * m;
            z* sv = t->sinv[l] + (long long)i * m * m;
            z* y1 = t->Y1[l] + (long long)i * m * (n1 + n2);
            z* y2 = t->Y2[l] + (long long)i * m * (n1 + n2);
            if (t->kform) {
                // [Y1; Y2] = M^-1 blockdiag(T1_iN, T2_iN), M = [[A1, nu I], [nu I, A2]]:
                //   Y1 = K^-1 [-A2 T1_iN, nu T2_iN],  Y2 = ([T1_iN, 0] - A1 Y1) / nu,  K = nu^2 I - A2 A1
                z* kv = t->kinv[l] + (long long)i * m * m;
                const ZView t1in = band_view(r1 + o1, ld, INT_MAX, 0, o1, m);
                const ZView t2in = band_view(r2 + o2, ld, INT_MAX, 0, o2, m);
                {   // K = nu^2 I - A2 A1
                    GemmDesc g = gdesc(m, m, m, zview(dv, m), zview(sv, m), zout(kv, m), mone);
                    g.C = zview(kv, m); g.beta = one;
                    mk.push_back(g);
                }
                // B1 = -A2 T1_iN, held in Y2's first n1 columns until Y2 is formed
                m1.push_back(gdesc(m, n1, m, zview(dv, m), t1in, zout(y2, m), mone));
                // Y1 = [K^-1 B1, nu K^-1 T2_iN]
                m2.push_back(gdesc(m, n1, m, zview(kv, m), zview(y2, m), zout(y1, m), one));
                m2.push_back(gdesc(m, n2, m, zview(kv, m), t2in, zout(y1 + (long long)m * n1, m), t->nu));
                {   // Y2 = (X1 - A1 Y1) / nu, X1 = [T1_iN, 0]
                    GemmDesc g = gdesc(m, n1, m, zview(sv, m), zview(y1, m), zout(y2, m), mrnu);
                    g.C = t1in; g.beta = rnu;
                    m3.push_back(g);
                    m3.push_back(gdesc(m, n2, m, zview(sv, m), zview(y1 + (long long)m * n1, m),
                                       zout(y2 + (long long)m * n1, m), mrnu));
                }
            } else {
            // Y2R = inv(D) T2_iN
            m1.push_back(gdesc(m, n2, m, zview(dv, m), band_view(r2 + o2, ld, INT_MAX, 0, o2, m),
                               zout(y2 + (long long)m * n1, m), one));
            // Y1L = inv(S) T1_iN ; Y1R = -nu inv(S) Y2R
            m2.push_back(gdesc(m, n1, m, zview(sv, m), band_view(r1 + o1, ld, INT_MAX, 0, o1, m), zout(y1, m), one));
            m2.push_back(gdesc(m, n2, m, zview(sv, m), zview(y2 + (long long)m * n1, m),
                               zout(y1 + (long long)m * n1, m), mnu));
            // Y2L = -nu inv(D) Y1L ; Y2R = Y2R - nu inv(D) Y1R
            m3.push_back(gdesc(m, n1, m, zview(dv, m), zview(y1, m), zout(y2, m), mnu));
            {
                GemmDesc g = gdesc(m, n2, m, zview(dv, m), zview(y1 + (long long)m * n1, m),
                                   zout(y2 + (long long)m * n1, m), mnu);
                g.C = zview(y2 + (long long)m * n1, m);
                g.beta = one;
                m3.push_back(g);
            }
            }
            if (!(l == 0 && t->skip_root)) {
                z* par = t->rtr[l] + (long long)i * p.nb * p.nb;
                const ZView t1ni = band_view(r1 + (long long)o1 * ld, ld, o1, m, INT_MAX, 0);
                const ZView t2ni = band_view(r2 + (long long)o2 * ld, ld, o2, m, INT_MAX, 0);
                ZOut o11 = zout(par, p.nb), o12 = zout(par, p.nb), o21 = zout(par, p.nb), o22 = zout(par, p.nb);
                o11.rmap = t->d_pmap1[l]; o11.cmap = t->d_pmap1[l];
                o12.rmap = t->d_pmap1[l]; o12.cmap = t->d_pmap2[l];
                o21.rmap = t->d_pmap2[l]; o21.cmap = t->d_pmap1[l];
                o22.rmap = t->d_pmap2[l]; o22.cmap = t->d_pmap2[l];
                GemmDesc g11 = gdesc(n1, n1, m, t1ni, zview(y1, m), o11, one);
                g11.C = band_view(r1, ld, o1, m, o1, m);
                g11.beta = one;
                GemmDesc g12 = gdesc(n1, n2, m, t1ni, zview(y1 + (long long)m * n1, m), o12, one);
                GemmDesc g21 = gdesc(n2, n1, m, t2ni, zview(y2, m), o21, one);
                GemmDesc g22 = gdesc(n2, n2, m, t2ni, zview(y2 + (long long)m * n1, m), o22, one);
                g22.C = band_view(r2, ld, o2, m, o2, m);
                g22.beta = one;
                m4.push_back(g11); m4.push_back(g12); m4.push_back(g21); m4.push_back(g22);
                if (split) {
                    // the same four products, each split by rows into the face and the other rows:
                    // T_a,Ni(rows, :) Y_b (+ T_a,NN(rows, :) when a = b), rows to pmap_a, columns to pmap_b
                    const int par_ = i & 1;
                    for (int kind = 0; kind < 2; ++kind)
                        for (int a = 0; a < 2; ++a)
                            for (int b2 = 0; b2 < 2; ++b2) {
                                const int rows = cnt[par_][a][kind];
                                if (rows == 0) continue;
                                const z* ra = a == 0 ? r1 : r2;
                                const int oa = a == 0 ? o1 : o2;
                                ZView A = zview(ra + (long long)oa * ld, ld);
                                A.rmap = d_sel[par_][a][kind];
                                const z* yb = (a == 0 ? y1 : y2) + (b2 == 0 ? 0LL : (long long)m * n1);
                                ZOut D = zout(par, p.nb);
                                D.rmap = d_out[par_][a][kind];
                                D.cmap = b2 == 0 ? t->d_pmap1[l] : t->d_pmap2[l];
                                GemmDesc g = gdesc(rows, b2 == 0 ? n1 : n2, m, A, zview(yb, m), D, one);
                                if (a == b2) {
                                    ZView C = band_view(ra, ld, INT_MAX, 0, oa, m);
                                    C.rmap = d_sel[par_][a][kind];
                                    g.C = C;
                                    g.beta = one;
                                }
                                (kind == 0 ? m4f : m4n).push_back(g);
                            }
                }
            }
        }
        if ((rc = upload_gemm(t, t->bufs, mk, t->fK[l]))) return rc;
        if ((rc = upload_gemm(t, t->bufs, m1, t->fM1[l]))) return rc;
        if ((rc = upload_gemm(t, t->bufs, m2, t->fM2[l]))) return rc;
        if ((rc = upload_gemm(t, t->bufs, m3, t->fM3[l]))) return rc;
        if ((rc = upload_gemm(t, t->bufs, m4, t->fM4[l]))) return rc;
        if ((rc = upload_gemm(t, t->bufs, m4f, t->fM4F[l]))) return rc;
        if ((rc = upload_gemm(t, t->bufs, m4n, t->fM4N[l]))) return rc;
    }
    t->factor_ready = true;
    return RB_OK;
}

#define RB_LAUNCH(call)                                                                          \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            t->err = std::string("CUDA launch failed: ") + cudaGetErrorString(e_) + " in " #call; \
            return RB_ERR_CUDA;                                                                  \
        }                                                                                        \
    } while (0)

#define RB_TIMED(name, flops, call)                                                              \
    do {                                                                                         \
        int rc_ = ltimer_begin(t, name, flops);                                                  \
        if (rc_) return rc_;                                                                     \
        RB_LAUNCH(call);                                                                         \
        if ((rc_ = ltimer_end(t))) return rc_;                                                   \
    } while (0)

// a GEMM batch, timed under the name of the engine it runs on
#define RB_GEMM(batch, stream) RB_TIMED(gemm_stage_name(batch), (batch).flops, launch_gemm_batch(batch, stream))

// merge level l of a mixed-precision factorization runs its GEMMs on the tcgen05 split-TF32
// kernel: below the top two levels, and only where the interface fills the 128-row MMA tile.
// Level L stands for the solve's leaf GEMM h = Y(:, nb:) f, which streams every leaf's Y once
// (HBM-bound): on the tensor cores in the mixed solve as well.
// With the int8 engine (the default) the tensor-core products are as accurate as the refinement
// needs from any of them, so a level goes to the tensor cores only where they are faster than the
// FP64 tiles: interfaces of at least 256 points (1024^2, L=12: levels 2-4; at m = 128 the digit
// passes and the 48-column tiles cost more than the FP64 products save).  Split TF32 keeps its
// 128-point rule.
// The top two merge levels (the root interface system) stay FP64, unless the tree was created
// with RB_FLAG_MIXED_INT8_TOP (int8 engine only): then their GEMMs run on the int8 engine too,
// and only their inversions stay FP64.
static bool mixed_top_levels(const rb_tree* t) {
    return t->mixed_int8_top && tc5_engine(GemmBatch{}) == TC5_ENGINE_INT8;
}
static bool mixed_level(const rb_tree* t, int l) {
    if (t->prec != RB_PREC_MIXED || (l < 2 && !mixed_top_levels(t))) return false;
    const int mmin = tc5_engine(GemmBatch{}) == TC5_ENGINE_INT8 ? 256 : 128;
    return l == t->P.L || t->P.lv[l].m >= mmin;
}
// Which factor stages of a mixed level run on the tcgen05 kernel: RB_MIXED_STAGES (read at every
// launch) is a bit mask over K = nu^2 I - A2 A1 (1), B1 (2), Y1 (4), Y2 (8) and the parent map
// (16).  The default leaves K (m^3, the smallest product of a level) on the FP64 tiles, which are
// as fast there; the int8 engine runs the rest.  The solve's batches follow their level.
static int mixed_stage_mask() {
    const char* v = std::getenv("RB_MIXED_STAGES");
    return v ? std::atoi(v) : 30;
}
static bool mixed_batch(const rb_tree* t, const GemmBatch& b, int l) {
    if (!mixed_level(t, l)) return false;
    if (l >= t->P.L) return true;
    int bit = 0;
    if (&b == &t->fK[l]) bit = 1;
    else if (&b == &t->fM1[l]) bit = 2;
    else if (&b == &t->fM2[l]) bit = 4;
    else if (&b == &t->fM3[l]) bit = 8;
    else if (&b == &t->fM4[l] || &b == &t->fM4F[l] || &b == &t->fM4N[l]) bit = 16;
    return bit == 0 || (mixed_stage_mask() & bit) != 0;
}
static cudaError_t launch_gemm_level(rb_tree* t, const GemmBatch& b, int l, cudaStream_t s) {
    return mixed_batch(t, b, l) ? launch_gemm_tc5(b, t->d_status, s) : launch_gemm_batch(b, s);
}
// The mixed solve applies its factor with the FP64 GEMMs: the sweeps' products are narrow (n =
// the right-hand sides), where the tcgen05 tile is slower than the FP64 one (1024^2, L=12, 32
// RHS: 21.4 against 26.2 ms for the refined solve), and the refinement's contraction is set by
// the factor's rounding, not the sweeps'.  RB_MIXED_SOLVE_ENGINE=tc5 (read at every solve) runs
// the sweeps' mixed levels on the tcgen05 kernel instead.
static bool mixed_solve_fp64() {
    const char* v = std::getenv("RB_MIXED_SOLVE_ENGINE");
    return !(v && std::strcmp(v, "tc5") == 0);
}
// Split-K plans of the mixed levels' factor stages, with two workspaces: B1 runs on the second
// stream beside K and its inverse, the other stages on the main stream.
static int ensure_mixed_factor_plan(rb_tree* t) {
    if (t->mixed_plan) return RB_OK;
    // one split-K workspace per stream that runs mixed-level GEMMs: the chain stream (K, Y1, Y2,
    // the face rows; in the serial schedule also the whole map), B1's stream, and the main stream's
    // remaining map rows of the pipelined schedule
    long long wmain = 0, wside = 0, wrest = 0;
    for (int l = 0; l < t->P.L; ++l) {
        if (!mixed_level(t, l)) continue;
        for (GemmBatch* b : {&t->fK[l], &t->fM2[l], &t->fM3[l], &t->fM4[l], &t->fM4F[l]})
            wmain = std::max(wmain, gemm_plan_split_tc5_factor(*b));
        wside = std::max(wside, gemm_plan_split_tc5_factor(t->fM1[l]));
        wrest = std::max(wrest, gemm_plan_split_tc5_factor(t->fM4N[l]));
    }
    // and one operand-plane workspace per stream (the tcgen05 kernel's split operands)
    size_t qmain = 0, qside = 0, qrest = 0;
    for (int l = 0; l < t->P.L; ++l) {
        if (!mixed_level(t, l)) continue;
        for (GemmBatch* b : {&t->fK[l], &t->fM2[l], &t->fM3[l], &t->fM4[l], &t->fM4F[l]})
            qmain = std::max(qmain, tc5_plane_bytes(*b));
        qside = std::max(qside, tc5_plane_bytes(t->fM1[l]));
        qrest = std::max(qrest, tc5_plane_bytes(t->fM4N[l]));
    }
    z* pm = nullptr;
    z* ps = nullptr;
    z* pr = nullptr;
    unsigned char *qm = nullptr, *qs = nullptr, *qr = nullptr;
    int rc;
    if (wmain > 0 && (rc = alloc_n(t, t->mixed_bufs, (size_t)wmain, &pm))) return rc;
    if (wside > 0 && (rc = alloc_n(t, t->mixed_bufs, (size_t)wside, &ps))) return rc;
    if (wrest > 0 && (rc = alloc_n(t, t->mixed_bufs, (size_t)wrest, &pr))) return rc;
    if (qmain > 0 && (rc = alloc_n(t, t->mixed_bufs, qmain, &qm))) return rc;
    if (qside > 0 && (rc = alloc_n(t, t->mixed_bufs, qside, &qs))) return rc;
    if (qrest > 0 && (rc = alloc_n(t, t->mixed_bufs, qrest, &qr))) return rc;
    for (int l = 0; l < t->P.L; ++l) {
        if (!mixed_level(t, l)) continue;
        for (GemmBatch* b : {&t->fK[l], &t->fM2[l], &t->fM3[l], &t->fM4[l], &t->fM4F[l]}) {
            if (b->t5_ksplit > 1) b->work = pm;
            b->t5_planes = qm;
            b->t5_plane_cap = qmain;
        }
        if (t->fM1[l].t5_ksplit > 1) t->fM1[l].work = ps;
        t->fM1[l].t5_planes = qs;
        t->fM1[l].t5_plane_cap = qside;
        if (t->fM4N[l].t5_ksplit > 1) t->fM4N[l].work = pr;
        t->fM4N[l].t5_planes = qr;
        t->fM4N[l].t5_plane_cap = qrest;
    }
    t->mixed_plan = true;
    return RB_OK;
}

#define RB_GEMM_L(batch, level, stream)                                                          \
    RB_TIMED(mixed_batch(t, batch, level) ? "zgemm_tc5" : gemm_stage_name(batch), (batch).flops,  \
             launch_gemm_level(t, batch, level, stream))

static double gj_flops(int m, int count) { return 8.0 * (double)m * m * m * count; }
// arithmetic of one structured leaf factor: b block inverses (8 a^3 each) and two block sweeps
// of S^T Z = C^T with nb right-hand sides (8 a^2 nb per block and sweep)
static double leaf_flops(const LeafGeom& g) {
    return 8.0 * g.a * g.a * g.a * g.b + 16.0 * g.a * g.a * (double)g.nb * g.b;
}

// The K-form merges, pipelined across levels (every untimed run; FP64 and mixed precision).
// Level l's parent map is formed in two row sets: the rows on the face its parent merges across
// (fM4F), which are all the parent's interface system reads (A1, A2 and K from the ii blocks, B1
// and Y1 from the iN blocks), and the other rows (fM4N).  The parent level's chain -- forms, K,
// its Gauss-Jordan inversion, Y1, Y2 and its own face rows -- runs on a second stream as soon as
// the face rows exist, beside the main stream's fM4N of the level below: the inversions, whose
// serial panel chains keep most SMs waiting, overlap the largest GEMMs of the step.  B1 runs on
// a third stream beside the inversion.  The two row sets of a map are disjoint, and no reader of
// a map's other rows starts before its fM4N (the parent's own map and the solve's sweep at that
// level wait for it); the root's map is formed whole, on the main stream, after the hook.
static bool factor_pipelined(const rb_tree* t) {
    static const bool off = [] {
        const char* v = std::getenv("RB_FACTOR_PIPELINE");
        return v && v[0] == '0';
    }();
    return !off && t->timing == 0 && t->kform && t->P.L >= 2;
}

static int run_merges_pipelined(rb_tree* t, const std::vector<cudaEvent_t>* rec,
                                const std::function<int()>* before_root_tail) {
    const Plan& P = t->P;
    const int L = P.L;
    cudaStream_t s = t->stream, c = t->stream2, s4 = t->stream4;
    int rc;
    RB_CK(cudaEventRecord(t->ev_face[L], s));            // the leaves' maps, whole
    RB_CK(cudaEventRecord(t->ev_rest[L], s));
    t->factor_was_pipelined = true;
    for (int l = L - 1; l >= 0; --l) {
        const PlanLevel& p = P.lv[l];
        const ChildStore cs = child_store(t, l);
        RB_CK(cudaStreamWaitEvent(c, t->ev_face[l + 1], 0));
        RB_LAUNCH(merge_form_d(cs, p.nnodes, p.m, p.o2, t->zeta, t->dinv[l], c));
        if (rec && l == 0) RB_CK(cudaEventRecord(t->ev_root_forms, c));
        RB_CK(cudaEventRecord(t->ev_d[l], c));
        RB_CK(cudaStreamWaitEvent(s4, t->ev_d[l], 0));
        RB_LAUNCH(launch_gemm_level(t, t->fM1[l], l, s4));          // B1 = -A2 T1_iN
        RB_CK(cudaEventRecord(t->ev_m1[l], s4));
        RB_LAUNCH(merge_form_s(cs, p.nnodes, p.m, p.o1, t->zeta, zmk(0.0, 0.0), t->dinv[l], t->sinv[l], c));
        RB_LAUNCH(merge_form_k(p.nnodes, p.m, t->nu, t->kinv[l], c));
        RB_LAUNCH(launch_gemm_level(t, t->fK[l], l, c));
        RB_LAUNCH(gj_invert_batch(t->gj_k[l].d_desc, p.nnodes, p.m, t->gj_work, t->d_status, c));
        // a solve's sweep at this level also waits for ev_rest[l + 1] (run_solve)
        if (rec) RB_CK(cudaEventRecord((*rec)[l], c));
        RB_CK(cudaStreamWaitEvent(c, t->ev_m1[l], 0));
        if (l == 0) {
            RB_CK(cudaStreamWaitEvent(c, t->ev_rest[1], 0));
            RB_CK(cudaEventRecord(t->ev_root_gj, c));
            RB_CK(cudaStreamWaitEvent(s, t->ev_root_gj, 0));   // joins both side streams
            if (before_root_tail && (rc = (*before_root_tail)())) return rc;
            RB_LAUNCH(launch_gemm_level(t, t->fM2[0], 0, s));
            RB_LAUNCH(launch_gemm_level(t, t->fM3[0], 0, s));
            RB_LAUNCH(launch_gemm_level(t, t->fM4[0], 0, s));
        } else {
            // Y1 and Y2 read only the children's face rows; this level's map reads them whole
            RB_LAUNCH(launch_gemm_level(t, t->fM2[l], l, c));
            RB_LAUNCH(launch_gemm_level(t, t->fM3[l], l, c));
            RB_CK(cudaEventRecord(t->ev_m3[l], c));
            RB_CK(cudaStreamWaitEvent(c, t->ev_rest[l + 1], 0));
            RB_LAUNCH(launch_gemm_level(t, t->fM4F[l], l, c));
            RB_CK(cudaEventRecord(t->ev_face[l], c));
            RB_CK(cudaStreamWaitEvent(s, t->ev_m3[l], 0));
            RB_LAUNCH(launch_gemm_level(t, t->fM4N[l], l, s));
            RB_CK(cudaEventRecord(t->ev_rest[l], s));
        }
    }
    return RB_OK;
}

// rec (optional): events recorded as the factor progresses, for a solve on another stream
// rec: progress events, one per level (the leaves at L), for a solve that overlaps the factor.
// before_root_tail: enqueued once the root's interface inverse is ready (and rec[0] recorded),
// ahead of the root's Y1, Y2 and own map, which then wait for it on the main stream.
static int run_factor(rb_tree* t, const z* dk, const std::vector<cudaEvent_t>* rec = nullptr,
                      const std::function<int()>* before_root_tail = nullptr) {
    const Plan& P = t->P;
    const int L = P.L, nl = P.nleaves();
    LeafGeom lg{P.leaf_a(), P.leaf_b(), P.leaf_nb(), P.leaf_n(), P.kb};
    cudaStream_t s = t->stream;
    int rc;
    RB_CK(cudaMemsetAsync(t->d_status, 0, sizeof(int), s));
    if ((rc = timer_begin(t, "leaf_factor"))) return rc;
    if (P.d == 2) {
        RB_TIMED("leaf_factor", leaf_flops(lg) * nl, leaf_block_factor(lg, nl, t->d_h, dk, t->leaf_sinv, t->leaf_Y,
                                                                        t->d_status, s));
    } else {
        // 3D: assemble every leaf's FD matrix, invert it (RTR_solve's zgetrf/zgetrs with an identity
        // right-hand side, robin_tree_module.f90:728-799), turn its face rows into Robin data
        const Leaf3Geom g3{P.leaf_a(), P.leaf_b(), P.leaf_c(), P.leaf_nb(), P.leaf_n(), P.kb};
        RB_TIMED("leaf_assemble", 0.0, leaf3_assemble(g3, nl, t->d_h, dk, t->leaf_sinv, s));
        RB_TIMED("gj_invert", gj_flops(g3.n, nl),
                 gj_invert_batch(t->gj_leaf.d_desc, nl, g3.n, t->leaf_gjwork, t->d_status, s));
        RB_TIMED("leaf_rtr", 0.0, leaf3_rtr(g3, nl, t->d_h, t->leaf_sinv, t->leaf_Y, s));
    }
    if ((rc = timer_end(t))) return rc;
    if (rec) RB_CK(cudaEventRecord((*rec)[L], s));
    t->factor_was_pipelined = false;
    if (factor_pipelined(t)) return run_merges_pipelined(t, rec, before_root_tail);
    static const char* lvl_names[] = {"merge_l0", "merge_l1", "merge_l2", "merge_l3", "merge_l4", "merge_l5",
                                      "merge_l6", "merge_l7", "merge_l8", "merge_l9", "merge_l10", "merge_l11",
                                      "merge_l12", "merge_l13", "merge_l14", "merge_l15", "merge_l16"};
    for (int l = L - 1; l >= 0; --l) {
        const PlanLevel& p = P.lv[l];
        const ChildStore cs = child_store(t, l);
        if ((rc = timer_begin(t, l < 17 ? lvl_names[l] : "merge_deep"))) return rc;
        if (t->kform) {
            // A2 = zeta I - T2_ii, A1 = zeta I - T1_ii; B1 = -A2 T1_iN on the second stream beside
            // K = nu^2 I - A2 A1 and its inversion
            RB_TIMED("merge_form", 0.0, merge_form_d(cs, p.nnodes, p.m, p.o2, t->zeta, t->dinv[l], s));
            if (rec && l == 0) RB_CK(cudaEventRecord(t->ev_root_forms, s));
            RB_TIMED("merge_form", 0.0, merge_form_s(cs, p.nnodes, p.m, p.o1, t->zeta, zmk(0.0, 0.0), t->dinv[l],
                                                     t->sinv[l], s));
            const bool fork = t->timing == 0;
            if (fork) {
                RB_CK(cudaEventRecord(t->ev_fork[l], s));
                RB_CK(cudaStreamWaitEvent(t->stream2, t->ev_fork[l], 0));
                RB_LAUNCH(launch_gemm_level(t, t->fM1[l], l, t->stream2));
                RB_CK(cudaEventRecord(t->ev_join[l], t->stream2));
            }
            RB_TIMED("merge_form", 0.0, merge_form_k(p.nnodes, p.m, t->nu, t->kinv[l], s));
            RB_GEMM_L(t->fK[l], l, s);
            RB_TIMED("gj_invert", gj_flops(p.m, p.nnodes),
                     gj_invert_batch(t->gj_k[l].d_desc, p.nnodes, p.m, t->gj_work, t->d_status, s));
            if (rec) RB_CK(cudaEventRecord((*rec)[l], s));      // inv(K), A1, A2 of level l are ready
            if (fork) RB_CK(cudaStreamWaitEvent(s, t->ev_join[l], 0));
            else RB_GEMM_L(t->fM1[l], l, s);
            if (l == 0 && before_root_tail && (rc = (*before_root_tail)())) return rc;
        } else {
            RB_TIMED("merge_form", 0.0, merge_form_d(cs, p.nnodes, p.m, p.o2, t->zeta, t->dinv[l], s));
            if (rec && l == 0) RB_CK(cudaEventRecord(t->ev_root_forms, s));
            RB_TIMED("gj_invert", gj_flops(p.m, p.nnodes), gj_invert_batch(t->gj_d[l].d_desc, p.nnodes, p.m, t->gj_work, t->d_status, s));
            // Y2R = inv(D) T2_iN needs only inv(D): on the second stream it overlaps the S inversion
            const bool fork = t->timing == 0;
            if (fork) {
                RB_CK(cudaEventRecord(t->ev_fork[l], s));
                RB_CK(cudaStreamWaitEvent(t->stream2, t->ev_fork[l], 0));
                RB_LAUNCH(launch_gemm_level(t, t->fM1[l], l, t->stream2));
                RB_CK(cudaEventRecord(t->ev_join[l], t->stream2));
            }
            RB_TIMED("merge_form", 0.0, merge_form_s(cs, p.nnodes, p.m, p.o1, t->zeta, t->nu, t->dinv[l], t->sinv[l], s));
            RB_TIMED("gj_invert", gj_flops(p.m, p.nnodes), gj_invert_batch(t->gj_s[l].d_desc, p.nnodes, p.m, t->gj_work, t->d_status, s));
            if (rec) RB_CK(cudaEventRecord((*rec)[l], s));      // inv(D), inv(S) of level l are ready
            if (fork) RB_CK(cudaStreamWaitEvent(s, t->ev_join[l], 0));
            else RB_GEMM_L(t->fM1[l], l, s);
            if (l == 0 && before_root_tail && (rc = (*before_root_tail)())) return rc;
        }
        RB_GEMM_L(t->fM2[l], l, s);
        RB_GEMM_L(t->fM3[l], l, s);
        RB_GEMM_L(t->fM4[l], l, s);
        if ((rc = timer_end(t))) return rc;
    }
    return RB_OK;
}

// ---------------------------------------------------------------------------------------------------
// cached solve plans (SolveSet): at most kMaxSolveSets besides the current one
constexpr size_t kMaxSolveSets = 8;
static void free_solve_set(rb_tree* t, SolveSet& c) {
    drop_graph(c.gx);
    free_list(t, c.bufs);
}
static void drop_solve_sets(rb_tree* t) {
    for (auto& c : t->solve_sets) free_solve_set(t, c);
    t->solve_sets.clear();
}
// frees the least recently used plans until at most `keep` remain
static void evict_solve_sets(rb_tree* t, size_t keep) {
    while (t->solve_sets.size() > keep) {
        size_t lru = 0;
        for (size_t i = 1; i < t->solve_sets.size(); ++i)
            if (t->solve_sets[i].used < t->solve_sets[lru].used) lru = i;
        free_solve_set(t, t->solve_sets[lru]);
        t->solve_sets.erase(t->solve_sets.begin() + (long)lru);
    }
}

static int ensure_solve_storage(rb_tree* t, int nrhs) {
    const Plan& P = t->P;
    const int L = P.L, nl = P.nleaves(), ab = P.leaf_interior(), nb = P.leaf_nb(), n = P.leaf_n();
    int rc;
    if (nrhs > t->cap_rhs) {
        if (t->d2h_pending) RB_CK(cudaStreamSynchronize(t->stream5));   // no read-back may still use sol
        drop_graph(t->gx_solve);
        t->gx_solve_rhs = 0;
        drop_solve_sets(t);                          // every cached plan points into the old buffers
        free_list(t, t->solve_desc_bufs);
        free_list(t, t->solve_bufs);
        t->solve_planes = nullptr;
        t->solve_planes_bytes = 0;
        t->built_rhs = 0;
        const int k = nrhs;
        if ((rc = alloc_n(t, t->solve_bufs, (size_t)k * nl * ab, &t->d_f))) return rc;
        t->hbuf.assign(L + 1, nullptr);
        t->gbuf.assign(L + 1, nullptr);
        size_t tmax = 0;
        for (int l = 0; l <= L; ++l) {
            const PlanLevel& p = P.lv[l];
            if (l > 0)
                if ((rc = alloc_n(t, t->solve_bufs, (size_t)p.nnodes * p.nb * k, &t->hbuf[l]))) return rc;
            if ((rc = alloc_n(t, t->solve_bufs, (size_t)p.nnodes * p.nb * k, &t->gbuf[l]))) return rc;
            if (l == 0 && L > 0) tmax = (size_t)p.nnodes * 2 * p.m * k;   // the root's x1, x2
        }
        if ((rc = alloc_n(t, t->solve_bufs, tmax, &t->tmp))) return rc;
        if ((rc = alloc_n(t, t->solve_bufs, (size_t)k * nl * n, &t->sol))) return rc;
        t->cap_rhs = k;
    }
    if (t->built_rhs == nrhs) return RB_OK;
    // keep the current count's plan, and take the requested count's from the cache if it is there
    if (t->built_rhs > 0) {
        SolveSet cur;
        cur.nrhs = t->built_rhs;
        cur.sL0 = t->sL0; cur.sLg = t->sLg; cur.sLf = t->sLf; cur.sR1 = t->sR1;
        cur.sF12 = t->sF12; cur.sF3 = t->sF3; cur.sF4 = t->sF4; cur.sF5 = t->sF5; cur.sBY = t->sBY;
        cur.bufs = std::move(t->solve_desc_bufs);
        t->solve_desc_bufs.clear();
        cur.gx = t->gx_solve_rhs == t->built_rhs ? t->gx_solve : nullptr;
        if (!cur.gx) drop_graph(t->gx_solve);
        cur.gx_launches = t->gx_solve_launches;
        cur.runs = cur.gx ? t->solve_runs : 0;
        cur.used = ++t->solve_clock;
        t->gx_solve = nullptr;
        t->solve_sets.push_back(std::move(cur));
    } else {
        drop_graph(t->gx_solve);
    }
    t->built_rhs = 0;
    t->gx_solve_rhs = 0;
    for (size_t i = 0; i < t->solve_sets.size(); ++i) {
        if (t->solve_sets[i].nrhs != nrhs) continue;
        SolveSet& c = t->solve_sets[i];
        t->sL0 = c.sL0; t->sLg = c.sLg; t->sLf = c.sLf; t->sR1 = c.sR1;
        t->sF12 = c.sF12; t->sF3 = c.sF3; t->sF4 = c.sF4; t->sF5 = c.sF5; t->sBY = c.sBY;
        t->solve_desc_bufs = std::move(c.bufs);
        t->gx_solve = c.gx;
        t->gx_solve_launches = c.gx_launches;
        t->solve_runs = c.runs;
        t->gx_solve_rhs = nrhs;
        t->solve_sets.erase(t->solve_sets.begin() + (long)i);
        t->built_rhs = nrhs;
        return RB_OK;
    }
    evict_solve_sets(t, kMaxSolveSets - 1);
    t->solve_runs = 0;
    // descriptor batches for this RHS count (their arrays in solve_desc_bufs)
    const int k = nrhs;
    const z one = zmk(1.0, 0.0), mone = zmk(-1.0, 0.0), mnu = zneg(t->nu);
    const z rnu = zrcp(t->nu), mrnu = zneg(rnu);
    std::vector<GemmDesc> v;
    for (int i = 0; i < nl; ++i)
        v.push_back(gdesc(nb, k, ab, zview(t->leaf_Y + (long long)i * nb * n + (long long)nb * nb, nb),
                          zview(t->d_f + (long long)i * ab, (long long)nl * ab),
                          zout(t->hbuf[L] + (long long)i * nb * k, nb), one));
    if ((rc = upload_gemm(t, t->solve_desc_bufs, v, t->sL0))) return rc;
    t->sLg = GemmBatch();
    t->sLf = GemmBatch();
    if (P.d == 3) {
        // the leaf solve of RTR_solve (u = A^-1 [g; f]) as two products with the stored inverse:
        // u = A^-1(:, :nb) g, then u += A^-1(:, nb:) f; u is [rhs][leaf][n], g [leaf][rhs][nb]
        std::vector<GemmDesc> vg, vf;
        for (int i = 0; i < nl; ++i) {
            const z* ainv = t->leaf_sinv + (long long)i * n * n;
            z* u = t->sol + (long long)i * n;
            vg.push_back(gdesc(n, k, nb, zview(ainv, n), zview(t->gbuf[L] + (long long)i * k * nb, nb),
                               zout(u, (long long)nl * n), one));
            GemmDesc gf = gdesc(n, k, ab, zview(ainv + (long long)nb * n, n),
                                zview(t->d_f + (long long)i * ab, (long long)nl * ab), zout(u, (long long)nl * n), one);
            gf.C = zview(u, (long long)nl * n);
            gf.beta = one;
            vf.push_back(gf);
        }
        if ((rc = upload_gemm(t, t->solve_desc_bufs, vg, t->sLg))) return rc;
        if ((rc = upload_gemm(t, t->solve_desc_bufs, vf, t->sLf))) return rc;
    }
    t->sF12.assign(L, GemmBatch()); t->sF3.assign(L, GemmBatch()); t->sF4.assign(L, GemmBatch());
    t->sF5.assign(L, GemmBatch()); t->sBY.assign(L, GemmBatch());
    t->sR1 = GemmBatch();
    for (int l = 0; l < L; ++l) {
        const PlanLevel& p = P.lv[l];
        const int m = p.m, n1 = p.n1, n2 = p.n2, o1 = p.o1, o2 = p.o2, nbc = p.nbc, nbp = p.nb;
        const ChildStore cs = child_store(t, l);
        std::vector<GemmDesc> f12, f3, f4, f5, by, rx;
        for (int i = 0; i < p.nnodes; ++i) {
            const z* r1 = cs.rtr + (2LL * i) * cs.stride;
            const z* r2 = cs.rtr + (2LL * i + 1) * cs.stride;
            const long long ld = cs.ld;
            z* dv = t->dinv[l] + (long long)i * m * m;
            z* sv = t->sinv[l] + (long long)i * m * m;
            z* h1 = t->hbuf[l + 1] + (2LL * i) * nbc * k;
            z* h2 = t->hbuf[l + 1] + (2LL * i + 1) * nbc * k;
            z* g1 = t->gbuf[l + 1] + (2LL * i) * nbc * k;
            z* g2 = t->gbuf[l + 1] + (2LL * i + 1) * nbc * k;
            // the root's forward and backward steps are one: (g1, g2) = M^-1 (x1, x2) with
            // x_i = h_i + T_iN g_N (the root's g_N is the boundary data), x in tmp
            const bool root = l == 0;
            z* tb = root ? t->tmp + (long long)i * 2 * m * k : nullptr;
            const ZView x1 = root ? zview(tb, m) : zview(h1 + o1, nbc);
            const ZView x2 = root ? zview(tb + (long long)m * k, m) : zview(h2 + o2, nbc);
            if (root) {
                GemmDesc gx1 = gdesc(m, k, n1, band_view(r1 + o1, ld, INT_MAX, 0, o1, m),
                                     band_view(g1, nbc, o1, m, INT_MAX, 0), zout(tb, m), one);
                gx1.C = zview(h1 + o1, nbc); gx1.beta = one;
                GemmDesc gx2 = gdesc(m, k, n2, band_view(r2 + o2, ld, INT_MAX, 0, o2, m),
                                     band_view(g2, nbc, o2, m, INT_MAX, 0), zout(tb + (long long)m * k, m), one);
                gx2.C = zview(h2 + o2, nbc); gx2.beta = one;
                rx.push_back(gx1); rx.push_back(gx2);
            }
            if (t->kform) {
                // (g1, g2) = M^-1 (x1, x2): t = nu x2 - A2 x1 (in g2), g1 = K^-1 t,
                // g2 = (x1 - A1 g1) / nu
                z* kv = t->kinv[l] + (long long)i * m * m;
                GemmDesc gt = gdesc(m, k, m, zview(dv, m), x1, zout(g2 + o2, nbc), mone);
                gt.C = x2; gt.beta = t->nu;
                f12.push_back(gt);
                f3.push_back(gdesc(m, k, m, zview(kv, m), zview(g2 + o2, nbc), zout(g1 + o1, nbc), one));
                GemmDesc g2d = gdesc(m, k, m, zview(sv, m), zview(g1 + o1, nbc), zout(g2 + o2, nbc), mrnu);
                g2d.C = x1; g2d.beta = rnu;
                f4.push_back(g2d);
            } else {
                // g2 = inv(D) x2 ; g1 = inv(S) x1
                f12.push_back(gdesc(m, k, m, zview(dv, m), x2, zout(g2 + o2, nbc), one));
                f12.push_back(gdesc(m, k, m, zview(sv, m), x1, zout(g1 + o1, nbc), one));
                {   // g1_i -= nu inv(S) g2_i
                    GemmDesc g = gdesc(m, k, m, zview(sv, m), zview(g2 + o2, nbc), zout(g1 + o1, nbc), mnu);
                    g.C = zview(g1 + o1, nbc); g.beta = one;
                    f3.push_back(g);
                }
                {   // g2_i -= nu inv(D) g1_i
                    GemmDesc g = gdesc(m, k, m, zview(dv, m), zview(g1 + o1, nbc), zout(g2 + o2, nbc), mnu);
                    g.C = zview(g2 + o2, nbc); g.beta = one;
                    f4.push_back(g);
                }
            }
            if (l > 0) {   // parent h = h_N + T_Ni g_i
                z* hp = t->hbuf[l] + (long long)i * nbp * k;
                ZOut oa = zout(hp, nbp), ob = zout(hp, nbp);
                oa.rmap = t->d_pmap1[l];
                ob.rmap = t->d_pmap2[l];
                GemmDesc ga = gdesc(n1, k, m, band_view(r1 + (long long)o1 * ld, ld, o1, m, INT_MAX, 0),
                                    zview(g1 + o1, nbc), oa, one);
                ga.C = band_view(h1, nbc, o1, m, INT_MAX, 0); ga.beta = one;
                GemmDesc gb = gdesc(n2, k, m, band_view(r2 + (long long)o2 * ld, ld, o2, m, INT_MAX, 0),
                                    zview(g2 + o2, nbc), ob, one);
                gb.C = band_view(h2, nbc, o2, m, INT_MAX, 0); gb.beta = one;
                f5.push_back(ga); f5.push_back(gb);
            }
            if (l > 0) {
                // backward below the root: the interface values are the forward's particular part
                // (already in g1, g2 at the interface) plus [Y1; Y2] g_N, g_N = the node's incoming
                // values at the children's outer points (pmap1, pmap2 into the node's face order)
                ZView gn = zview(t->gbuf[l] + (long long)i * nbp * k, nbp);
                gn.rmap = t->d_pmapc[l];
                GemmDesc gy1 = gdesc(m, k, n1 + n2, zview(t->Y1[l] + (long long)i * m * (n1 + n2), m), gn,
                                     zout(g1 + o1, nbc), one);
                gy1.C = zview(g1 + o1, nbc); gy1.beta = one;
                GemmDesc gy2 = gdesc(m, k, n1 + n2, zview(t->Y2[l] + (long long)i * m * (n1 + n2), m), gn,
                                     zout(g2 + o2, nbc), one);
                gy2.C = zview(g2 + o2, nbc); gy2.beta = one;
                by.push_back(gy1); by.push_back(gy2);
            }
        }
        if ((rc = upload_gemm(t, t->solve_desc_bufs, f12, t->sF12[l]))) return rc;
        if ((rc = upload_gemm(t, t->solve_desc_bufs, f3, t->sF3[l]))) return rc;
        if ((rc = upload_gemm(t, t->solve_desc_bufs, f4, t->sF4[l]))) return rc;
        if ((rc = upload_gemm(t, t->solve_desc_bufs, f5, t->sF5[l]))) return rc;
        if ((rc = upload_gemm(t, t->solve_desc_bufs, by, t->sBY[l]))) return rc;
        if (l == 0 && (rc = upload_gemm(t, t->solve_desc_bufs, rx, t->sR1))) return rc;
    }
    t->sL0.fixed_order = true;
    t->sR1.fixed_order = true;
    t->sLg.fixed_order = true;
    t->sLf.fixed_order = true;
    for (int l = 0; l < L; ++l)
        for (GemmBatch* gb : {&t->sF12[l], &t->sF3[l], &t->sF4[l], &t->sF5[l], &t->sBY[l]}) gb->fixed_order = true;
    // split-K for the long-k, few-CTA solve GEMMs; one workspace serves them all (one stream)
    {
        std::vector<GemmBatch*> all{&t->sL0, &t->sR1};
        if (P.d == 3) { all.push_back(&t->sLg); all.push_back(&t->sLf); }
        for (int l = 0; l < L; ++l)
            for (GemmBatch* gb : {&t->sF12[l], &t->sF3[l], &t->sF4[l], &t->sF5[l], &t->sBY[l]}) all.push_back(gb);
        long long wmax = 0;
        for (GemmBatch* gb : all) {
            wmax = std::max(wmax, gemm_plan_split(*gb));
            wmax = std::max(wmax, gemm_plan_split_tc5(*gb));     // the same batch on tcgen05 (mixed)
        }
        if (wmax > 0) {
            z* ws = nullptr;
            if ((rc = alloc_n(t, t->solve_desc_bufs, (size_t)wmax, &ws))) return rc;
            for (GemmBatch* gb : all)
                if (gb->ksplit > 1 || gb->t5_ksplit > 1) gb->work = ws;
        }
    }
    t->built_rhs = nrhs;
    t->gx_solve_rhs = nrhs;
    return RB_OK;
}

// The solve on stream s.  wait (optional): the factor's progress events (run_factor's rec); the
// leaf forward GEMM waits for the leaves and forward level l for level l of a factor that runs
// on another stream; the backward sweep reads only levels the forward sweep waited for.
// out: where the leaf solutions go (t->sol when null).  inject: subtract the interface rows of
// the residual (t->d_ri) from the children's outgoing data before each level's merge (the
// correction sweeps of the mixed-precision refinement).
// Operand planes of the solve batches that run on the tcgen05 kernel (RB_MIXED_SOLVE_ENGINE=tc5):
// one workspace for them all (the sweep is one stream), grown on first use.
static int ensure_solve_planes(rb_tree* t) {
    const int L = t->P.L;
    std::vector<GemmBatch*> mixed;
    if (mixed_level(t, L)) mixed.push_back(&t->sL0);
    for (int l = 1; l < L; ++l)
        if (mixed_level(t, l))
            for (GemmBatch* gb : {&t->sF12[l], &t->sF3[l], &t->sF4[l], &t->sF5[l], &t->sBY[l]}) mixed.push_back(gb);
    size_t need = 0;
    for (GemmBatch* gb : mixed) need = std::max(need, tc5_plane_bytes(*gb));
    if (need > t->solve_planes_bytes) {
        unsigned char* q = nullptr;
        int rc = alloc_n(t, t->solve_bufs, need, &q);
        if (rc) return rc;
        t->solve_planes = q;
        t->solve_planes_bytes = need;
    }
    for (GemmBatch* gb : mixed) {
        gb->t5_planes = t->solve_planes;
        gb->t5_plane_cap = t->solve_planes_bytes;
    }
    return RB_OK;
}

// the solution buffer is about to be written on stream s: wait (on the device) for the read-backs
// rb_get_solution_async enqueued from it.  Inside a stream capture the wait is not recorded: a
// graphed solve waits before its graph is launched (solve_common).
static int wait_readback(rb_tree* t, cudaStream_t s) {
    if (!t->d2h_pending) return RB_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    RB_CK(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusNone) RB_CK(cudaStreamWaitEvent(s, t->ev_d2h, 0));
    return RB_OK;
}

static int run_solve(rb_tree* t, int k, cudaStream_t s, const std::vector<cudaEvent_t>* wait = nullptr,
                     z* out = nullptr, bool inject = false) {
    const Plan& P = t->P;
    const int L = P.L, nl = P.nleaves();
    LeafGeom lg{P.leaf_a(), P.leaf_b(), P.leaf_nb(), P.leaf_n(), P.kb};
    int rc;
    const bool sweep_fp64 = mixed_solve_fp64();
    if (!sweep_fp64 && t->prec == RB_PREC_MIXED && (rc = ensure_solve_planes(t))) return rc;
#define RB_GEMM_S(batch, level, stream)                                                          \
    do {                                                                                         \
        if (sweep_fp64) RB_GEMM(batch, stream);                                                  \
        else RB_GEMM_L(batch, level, stream);                                                    \
    } while (0)
    auto inject_level = [&](int l) -> int {
        if (!inject) return RB_OK;
        const PlanLevel& p = P.lv[l];
        RB_TIMED("sweep_aux", 0.0, iface_inject(p.nnodes, p.m, p.nbc, p.o1, p.o2, k, nl * P.leaf_nb(), t->d_ifrows[l],
                                                t->d_ri, t->hbuf[l + 1], s));
        return RB_OK;
    };
    if ((rc = timer_begin(t, "forward"))) return rc;
    if (wait) RB_CK(cudaStreamWaitEvent(s, (*wait)[L], 0));
    RB_GEMM_S(t->sL0, L, s);
    for (int l = L - 1; l >= 1; --l) {
        if (wait) RB_CK(cudaStreamWaitEvent(s, (*wait)[l], 0));
        // a pipelined factor records level l's event after the inversion, before the children's
        // maps are whole; the parent h of this level reads their non-interface rows
        if (wait && t->factor_was_pipelined) RB_CK(cudaStreamWaitEvent(s, t->ev_rest[l + 1], 0));
        if ((rc = inject_level(l))) return rc;
        RB_GEMM_S(t->sF12[l], l, s);
        RB_GEMM_S(t->sF3[l], l, s);
        RB_GEMM_S(t->sF4[l], l, s);
        RB_GEMM_S(t->sF5[l], l, s);
    }
    // the root: x = h + T_iN g_N needs level 1's maps (and the K form's first product, A2), not
    // the root's inverse, so it runs as soon as the root's A2 is formed
    if (L > 0) {
        const PlanLevel& p = P.lv[0];
        if (wait) RB_CK(cudaStreamWaitEvent(s, t->ev_root_forms, 0));
        if ((rc = inject_level(0))) return rc;
        RB_TIMED("sweep_aux", 0.0, sweep_scatter_down(p.nnodes, k, p.nb, p.nbc, p.m, p.o1, p.o2, p.n1, p.n2,
                                                      t->d_pmap1[0], t->d_pmap2[0], t->gbuf[0], t->gbuf[1], s));
        RB_GEMM(t->sR1, s);
        if (t->kform) RB_GEMM(t->sF12[0], s);
        if (wait) RB_CK(cudaStreamWaitEvent(s, (*wait)[0], 0));
        if (!t->kform) RB_GEMM(t->sF12[0], s);
        RB_GEMM(t->sF3[0], s);
        RB_GEMM(t->sF4[0], s);
    }
    if ((rc = timer_end(t))) return rc;
    if ((rc = timer_begin(t, "backward"))) return rc;
    for (int l = 1; l < L; ++l) {
        const PlanLevel& p = P.lv[l];
        RB_TIMED("sweep_aux", 0.0, sweep_scatter_down(p.nnodes, k, p.nb, p.nbc, p.m, p.o1, p.o2, p.n1, p.n2, t->d_pmap1[l],
                                     t->d_pmap2[l], t->gbuf[l], t->gbuf[l + 1], s));
        RB_GEMM_S(t->sBY[l], l, s);
    }
    if ((rc = timer_end(t))) return rc;
    if ((rc = timer_begin(t, "leaf_recover"))) return rc;
    if ((!out || out == t->sol) && (rc = wait_readback(t, s))) return rc;
    if (P.d == 2) {
        RB_TIMED("leaf_solve", 0.0, leaf_block_solve(lg, nl, k, t->d_h, t->d_f, t->gbuf[L], t->leaf_sinv,
                                                     out ? out : t->sol, s));
    } else {
        if (out && out != t->sol) return fail(t, RB_ERR_UNSUPPORTED, "3D leaf solve into a second buffer");
        RB_GEMM(t->sLg, s);
        RB_GEMM(t->sLf, s);
    }
    if ((rc = timer_end(t))) return rc;
    return RB_OK;
#undef RB_GEMM_S
}

// ---------------------------------------------------------------------------------------------------
// Mixed-precision refinement: tables of the global FD system's boundary rows and the loop.

// bclass[leaf*nb + r]: the root boundary position of a point on the domain boundary, or
// -1 - (leaf'*nb + r') of the neighbouring leaf's row for the same interface point; ifrows[l]:
// for every node of level l and child k, the leaf boundary rows of the child's interface points
// in the child's face order.  Both follow the merges' face orderings (pmap1, pmap2) from the
// leaves up, so the interface rows land where each merge reads its children's outgoing data.
static std::string build_refine_tables(const Plan& P, std::vector<int>& bclass, std::vector<std::vector<int>>& ifrows) {
    const int L = P.L;
    const PlanLevel& lf = P.lv[L];
    const int nl = lf.nnodes, nb = lf.nb;
    std::vector<int> cur((size_t)nl * nb);
    for (size_t e = 0; e < cur.size(); ++e) cur[e] = (int)e;
    ifrows.assign(L, {});
    for (int l = L - 1; l >= 0; --l) {
        const PlanLevel& p = P.lv[l];
        const PlanLevel& c = P.lv[l + 1];
        std::vector<int> par((size_t)p.nnodes * p.nb, -1);
        std::vector<int>& ir = ifrows[l];
        ir.assign((size_t)p.nnodes * 2 * p.m, -1);
        for (int i = 0; i < p.nnodes; ++i)
            for (int k = 0; k < 2; ++k) {
                const int child = 2 * i + k, o = k ? p.o2 : p.o1;
                const std::vector<int>& pm = k ? p.pmap2 : p.pmap1;
                for (int q = 0; q < (int)pm.size(); ++q) {
                    const int phys = q < o ? q : q + p.m;
                    par[(size_t)i * p.nb + pm[q]] = cur[(size_t)child * c.nb + phys];
                }
                for (int q = 0; q < p.m; ++q) ir[((size_t)i * 2 + k) * p.m + q] = cur[(size_t)child * c.nb + o + q];
            }
        cur.swap(par);
    }
    bclass.assign((size_t)nl * nb, INT_MIN);
    for (int q = 0; q < (int)cur.size(); ++q) {
        if (cur[q] < 0) return "refinement tables: root boundary point without a leaf row";
        bclass[cur[q]] = q;
    }
    // interface points: the neighbour across each inner face, found by exact box coordinates
    // (every box edge is produced by the same bisection arithmetic on both sides)
    std::map<std::pair<double, double>, int> by_lo, by_hix, by_hiy;
    for (int i = 0; i < nl; ++i) {
        const double* lo = &lf.lo[3 * i];
        const double* hi = &lf.hi[3 * i];
        by_lo[{lo[0], lo[1]}] = i;
        by_hix[{hi[0], lo[1]}] = i;
        by_hiy[{lo[0], hi[1]}] = i;
    }
    for (int i = 0; i < nl; ++i) {
        const double* lo = &lf.lo[3 * i];
        const double* hi = &lf.hi[3 * i];
        for (int f = 0; f < 4; ++f) {
            if (lf.isb[P.nf() * i + f]) continue;
            std::map<std::pair<double, double>, int>::const_iterator it;
            int fo;
            if (f == 0) { it = by_hix.find({lo[0], lo[1]}); fo = 1; if (it == by_hix.end()) return "refinement tables: no x1 neighbour"; }
            else if (f == 1) { it = by_lo.find({hi[0], lo[1]}); fo = 0; if (it == by_lo.end()) return "refinement tables: no x2 neighbour"; }
            else if (f == 2) { it = by_hiy.find({lo[0], lo[1]}); fo = 3; if (it == by_hiy.end()) return "refinement tables: no y1 neighbour"; }
            else { it = by_lo.find({lo[0], hi[1]}); fo = 2; if (it == by_lo.end()) return "refinement tables: no y2 neighbour"; }
            const int j = it->second;
            for (int q = 0; q < lf.pf[f]; ++q)
                bclass[(size_t)i * nb + lf.off[f] + q] = -1 - (j * nb + lf.off[fo] + q);
        }
    }
    for (int v : bclass)
        if (v == INT_MIN) return "refinement tables: a leaf boundary row is neither on the domain boundary nor on an interface";
    return "";
}

static int ensure_refine_storage(rb_tree* t, int k) {
    const Plan& P = t->P;
    int rc;
    if (!t->d_bclass) {
        const std::string msg = build_refine_tables(P, t->h_bclass, t->h_ifrows);
        if (!msg.empty()) return fail(t, RB_ERR_GEOMETRY, msg);
        if ((rc = alloc_n(t, t->bufs, t->h_bclass.size(), &t->d_bclass))) return rc;
        RB_CK(cudaMemcpy(t->d_bclass, t->h_bclass.data(), t->h_bclass.size() * sizeof(int), cudaMemcpyHostToDevice));
        t->d_ifrows.assign(P.L, nullptr);
        for (int l = 0; l < P.L; ++l) {
            if ((rc = alloc_n(t, t->bufs, t->h_ifrows[l].size(), &t->d_ifrows[l]))) return rc;
            RB_CK(cudaMemcpy(t->d_ifrows[l], t->h_ifrows[l].data(), t->h_ifrows[l].size() * sizeof(int),
                             cudaMemcpyHostToDevice));
        }
    }
    if (k > t->refine_cap) {
        free_list(t, t->refine_bufs);
        t->refine_cap = 0;
        const size_t per = (size_t)P.nleaves() * P.leaf_n();
        if ((rc = alloc_n(t, t->refine_bufs, per * k, &t->dsol))) return rc;
        if ((rc = alloc_n(t, t->refine_bufs, (size_t)P.nleaves() * P.leaf_nb() * k, &t->d_ri))) return rc;
        if ((rc = alloc_n(t, t->refine_bufs, (size_t)3 * k + 1, &t->d_norms))) return rc;
        if (t->h_norms) cudaFreeHost(t->h_norms);
        t->h_norms = nullptr;
        RB_CK(cudaMallocHost(&t->h_norms, ((size_t)3 * k + 1) * sizeof(double)));
        t->refine_cap = k;
    }
    return RB_OK;
}

// The mixed-precision solve of the k right-hand sides in t->d_f / t->gbuf[0]: a first sweep,
// then corrections d = M^-1 r with r = b - A x in FP64 until every right-hand side's estimated
// relative error is below refine_tol.  The error of x after adding d is about rho |d|, rho the
// contraction of the iteration (|d| / |x| for the first correction, |d| / |d_previous| after),
// so the loop stops when rho |d| <= tol |x| / 10.  The residual overwrites d_f and gbuf[0].
// wait (optional): the factor's progress events; the first sweep then runs beside the factor
// (run_solve's overlap), and the corrections after it.
static int refine_solve(rb_tree* t, int k, cudaStream_t s, const std::vector<cudaEvent_t>* wait = nullptr) {
    const Plan& P = t->P;
    int rc;
    if ((rc = ensure_refine_storage(t, k))) return rc;
    const size_t per = (size_t)P.nleaves() * P.leaf_n();
    RefineGeom rg{P.leaf_a(), P.leaf_b(), P.nleaves(), P.lv[0].nb, P.kb, t->zeta, t->nu};
    if ((rc = run_solve(t, k, s, wait, t->sol, false))) return rc;
    std::vector<double> dprev(k, 0.0), xn(k, 0.0);
    t->refine_iters = 0;
    t->refine_rho = 0.0;
    t->refine_est = 0.0;
    t->refine_res = 0.0;
    bool converged = false;
    for (int it = 0; it < t->refine_maxit; ++it) {
        RB_CK(cudaMemsetAsync(t->d_norms, 0, ((size_t)3 * k + 1) * sizeof(double), s));
        RB_TIMED("fd_residual", 0.0, fd_residual(rg, k, it == 0 ? t->sol : t->dsol, t->d_f, t->gbuf[0], t->d_ri, t->d_k,
                                                 t->d_h, t->d_bclass, it == 0, t->d_norms, s));
        if ((rc = run_solve(t, k, s, nullptr, t->dsol, true))) return rc;
        RB_TIMED("refine_update", 0.0, refine_update(t->sol, t->dsol, (long long)per, k, t->d_norms + k,
                                                     t->d_norms + 2 * k, s));
        RB_CK(cudaMemcpyAsync(t->d_norms + 3 * k, t->d_status, sizeof(int), cudaMemcpyDeviceToDevice, s));
        RB_CK(cudaMemcpyAsync(t->h_norms, t->d_norms, ((size_t)3 * k + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
        RB_CK(cudaStreamSynchronize(s));
        int st = 0;
        std::memcpy(&st, t->h_norms + 3 * k, sizeof(int));
        if (st & (RB_STATUS_GJ_TIMEOUT | RB_TC5_TIMEOUT))
            return fail(t, RB_ERR_CUDA, "a device wait timed out during the solve");
        t->refine_iters = it + 1;
        double worst = 0.0, rho_max = 0.0, res = 0.0;
        bool diverging = false;
        for (int r = 0; r < k; ++r) {
            const double rn = t->h_norms[r], x = t->h_norms[k + r], d = t->h_norms[2 * k + r];
            const double ref = it == 0 ? x : dprev[r];
            const double rho = ref > 0.0 ? d / ref : 0.0;
            const double rel = x > 0.0 ? d / x : 0.0;
            dprev[r] = d;
            xn[r] = x;
            res = std::max(res, x > 0.0 ? rn / x : 0.0);
            // a correction far below the tolerance: converged, whatever the ratio of two
            // rounding-level corrections says
            if (rel <= 1e-3 * t->refine_tol) continue;
            if (!(rho < 0.5)) diverging = true;
            rho_max = std::max(rho_max, rho);
            worst = std::max(worst, rho * rel);
        }
        t->refine_rho = std::max(t->refine_rho, rho_max);
        t->refine_est = worst;
        t->refine_res = res;
        if (!std::isfinite(worst) || diverging)
            return fail(t, RB_ERR_NUMERIC, "iterative refinement of the mixed-precision solve does not converge "
                                           "(contraction " + std::to_string(rho_max) + ")");
        if (worst <= 0.1 * t->refine_tol) {
            converged = true;
            break;
        }
    }
    if (!converged)
        return fail(t, RB_ERR_NUMERIC, "iterative refinement reached " + std::to_string(t->refine_maxit) +
                                           " corrections without meeting the tolerance (estimated error " +
                                           std::to_string(t->refine_est) + ")");
    return RB_OK;
}

// ---------------------------------------------------------------------------------------------------
// persistent leaf storage of a plan in bytes: the leaf factors (2D: b blocks of a x a; 3D: the
// dense n x n inverse), Y = R A^-1 and the potential samples
static double leaf_factor_bytes(const Plan& Q) {
    const double nint = (double)Q.leaf_interior(), n = (double)Q.leaf_n();
    const double fac = Q.d == 2 ? (double)Q.leaf_b() * Q.leaf_a() * Q.leaf_a() : n * n;
    return (double)Q.nleaves() * (fac + (double)Q.leaf_nb() * n + nint) * 16.0;
}

extern "C" {

int rb_tree_create(const rb_geom* geom, rb_tree** out) {
    if (!geom || !out) {
        g_create_error = "rb_tree_create: null argument";
        return RB_ERR_INVALID;
    }
    *out = nullptr;
    Plan P;
    std::string msg = build_plan(geom->d, geom->L, geom->domain, geom->h_tgt, geom->kb, P);
    if (!msg.empty()) {
        g_create_error = msg;
        if (geom->d == 3 && msg.find("not implemented") != std::string::npos) return RB_ERR_UNSUPPORTED;
        if (msg.find("Interface sizes") != std::string::npos) return RB_ERR_GEOMETRY;
        if (msg.find("Dimension") != std::string::npos || msg.find("domain") != std::string::npos) return RB_ERR_DOMAIN;
        return RB_ERR_INVALID;
    }
    if (geom->ordering != 1) {
        g_create_error = "Invalid ordering parameter in igrid2lin";
        return RB_ERR_INVALID;
    }
    // the batched Gauss-Jordan inversions hold matrices of up to 1024 rows: every interface and,
    // in 3D, every dense leaf
    for (int l = 0; l < P.L; ++l)
        if (P.lv[l].m > 1024) {
            g_create_error = "interface of " + std::to_string(P.lv[l].m) + " points on level " + std::to_string(l) +
                             ": interface inverses of more than 1024 points are not implemented";
            return RB_ERR_UNSUPPORTED;
        }
    if (P.d == 3 && P.leaf_n() > 1024) {
        g_create_error = "3D leaf of " + std::to_string(P.leaf_n()) +
                         " unknowns: dense leaf inverses of more than 1024 unknowns are not implemented";
        return RB_ERR_UNSUPPORTED;
    }
    // bndry_params(i,j) column-major, interleaved
    const double* bp = geom->bndry_params;
    const z b11 = zmk(bp[0], bp[1]), b21 = zmk(bp[2], bp[3]), b12 = zmk(bp[4], bp[5]), b22 = zmk(bp[6], bp[7]);
    const z det = zsub(zmul(b11, b22), zmul(b12, b21));
    if (std::hypot(det.x, det.y) < 1.0e-3) {
        g_create_error = "Error: Boundary parameter matrix is nearly singular.";
        return RB_ERR_BNDRY_PARAMS;
    }
    rb_tree* t = new rb_tree();
    t->geom = *geom;
    t->P = std::move(P);
    // nu and zeta of compute_RTR (robin_tree_module.f90:425-431)
    const z den = zmul(zmul(zmk(2.0, 0.0), b11), b12);
    const z rden = zrcp(den);
    t->nu = zmul(zadd(zneg(zmul(b11, b22)), zmul(b12, b21)), rden);
    t->zeta = zmul(zadd(zmul(b11, b22), zmul(b12, b21)), rden);
    // one inversion per merge (K = nu^2 I - A2 A1) unless nu is small against zeta, where the
    // division by nu in Y2 = (X1 - A1 Y1) / nu would lose digits; then inv(D) and inv(S)
    {
        const double an = std::sqrt(t->nu.x * t->nu.x + t->nu.y * t->nu.y);
        const double az = std::sqrt(t->zeta.x * t->zeta.x + t->zeta.y * t->zeta.y);
        t->kform = !(geom->flags & RB_FLAG_MERGE_DS) && an >= 0.1 * std::max(1.0, az);
    }
    t->budget = geom->device_budget;
    t->verbose = (geom->flags & RB_FLAG_VERBOSE) != 0;
    t->skip_root = (geom->flags & RB_FLAG_SKIP_ROOT_RTR) != 0;
    t->graphs = (geom->flags & RB_FLAG_NO_GRAPHS) == 0;
    t->async_factor = (geom->flags & RB_FLAG_ASYNC_FACTOR) != 0;
    t->mixed_int8_top = (geom->flags & RB_FLAG_MIXED_INT8_TOP) != 0;
    // refuse up front a problem the budget cannot hold (persistent factor storage only)
    if (t->budget > 0) {
        const Plan& Q = t->P;
        double need = leaf_factor_bytes(Q);
        for (int l = 0; l < Q.L; ++l)
            need += (double)Q.lv[l].nnodes *
                    ((double)Q.lv[l].nb * Q.lv[l].nb + (t->kform ? 3.0 : 2.0) * Q.lv[l].m * Q.lv[l].m +
                     2.0 * Q.lv[l].m * (Q.lv[l].n1 + Q.lv[l].n2)) * 16.0;
        if (need > (double)t->budget) {
            g_create_error = "device budget exceeded: the factorization needs at least " +
                             std::to_string((long long)need) + " bytes, budget " + std::to_string(t->budget);
            delete t;
            return RB_ERR_OUT_OF_MEMORY;
        }
    }
    if (t->verbose) std::printf("Domain partition completed.\n");
    *out = t;
    return RB_OK;
}

int rb_tree_destroy(rb_tree* t) {
    if (!t) return RB_OK;
    if (t->stream) cudaStreamSynchronize(t->stream);
    timers_collect(t);
    drop_graph(t->gx_factor);
    drop_graph(t->gx_solve);
    drop_solve_sets(t);
    free_list(t, t->solve_desc_bufs);
    free_list(t, t->solve_bufs);
    free_list(t, t->refine_bufs);
    free_list(t, t->mixed_bufs);
    free_list(t, t->bufs);
    if (t->h_norms) cudaFreeHost(t->h_norms);
    for (auto& e : t->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : t->ev_pool) cudaEventDestroy(e);
    for (auto& e : t->ev_fork) if (e) cudaEventDestroy(e);
    for (auto& e : t->ev_join) if (e) cudaEventDestroy(e);
    for (auto& e : t->ev_lvl) if (e) cudaEventDestroy(e);
    for (auto* v : {&t->ev_face, &t->ev_rest, &t->ev_d, &t->ev_m1, &t->ev_m3})
        for (auto& e : *v) if (e) cudaEventDestroy(e);
    if (t->ev_root_gj) cudaEventDestroy(t->ev_root_gj);
    if (t->ev_root_forms) cudaEventDestroy(t->ev_root_forms);
    if (t->stream3) cudaStreamSynchronize(t->stream3);
    if (t->ev_copy) cudaEventDestroy(t->ev_copy);
    if (t->h_status) cudaFreeHost(t->h_status);
    if (t->stream5) {
        cudaStreamSynchronize(t->stream5);
        cudaStreamDestroy(t->stream5);
    }
    if (t->ev_d2h) cudaEventDestroy(t->ev_d2h);
    if (t->stream3) cudaStreamDestroy(t->stream3);
    if (t->stream2) cudaStreamDestroy(t->stream2);
    if (t->stream4) cudaStreamDestroy(t->stream4);
    if (t->stream) cudaStreamDestroy(t->stream);
    delete t;
    return RB_OK;
}

const char* rb_last_error(const rb_tree* t) { return t ? t->err.c_str() : g_create_error.c_str(); }

int rb_tree_info(const rb_tree* t, rb_info* info) {
    if (!t || !info) return RB_ERR_INVALID;
    const Plan& P = t->P;
    info->nleaves = P.nleaves();
    info->leaf_a = P.leaf_a();
    info->leaf_b = P.leaf_b();
    info->leaf_n = P.leaf_n();
    info->leaf_nb = P.leaf_nb();
    info->root_nb = P.lv[0].nb;
    info->root_a = P.lv[0].a;
    info->root_b = P.lv[0].b;
    for (int j = 0; j < 3; ++j) info->h_last[j] = P.h_last[j];
    info->n_interior = (int64_t)P.nleaves() * P.leaf_interior();
    info->d = P.d;
    info->leaf_c = P.leaf_c();
    info->root_c = P.lv[0].c;
    info->reserved = 0;
    info->device_bytes = t->held;
    info->factored = t->factored ? 1 : 0;
    info->nrhs = t->nrhs;
    return RB_OK;
}

int rb_tree_sample_points(const rb_tree* t, int which, double* xyz) {
    if (!t || !xyz) return RB_ERR_INVALID;
    const Plan& P = t->P;
    const PlanLevel& lf = P.lv[P.L];
    const int a = lf.a, b = lf.b, c = lf.c, nl = lf.nnodes, d = P.d;
    // grid2real (fd_module.f90:669-700): lo + g*h - h/2, snapped to the face on the boundary; in 2D
    // the third coordinate is lo_z (gk = 1, h_z = 0)
    auto coord = [&](int leaf, int gi, int gj, int gk, const double* h, double* out) {
        const double* lo = &lf.lo[3 * leaf];
        const double* hi = &lf.hi[3 * leaf];
        const int g[3] = {gi, gj, gk}, sh[3] = {a, b, c};
        for (int ax = 0; ax < 3; ++ax) {
            out[ax] = (lo[ax] + g[ax] * h[ax]) - h[ax] / 2;
            if (ax < d) {
                if (g[ax] == 0) out[ax] = lo[ax];
                else if (g[ax] == sh[ax] + 1) out[ax] = hi[ax];
            }
        }
    };
    // the points of face f (0-based) of a leaf in the face's own order (lin2fgrid,
    // fd_module.f90:867-939): the first tangential index fastest
    auto face_grid = [&](int f, int s1, int s2, int* g) {
        const int ax = f / 2, fix = (f % 2 == 0) ? 0 : (ax == 0 ? a : ax == 1 ? b : c) + 1;
        int tang[2], q = 0;
        for (int k = 0; k < 3; ++k)
            if (k != ax) tang[q++] = k;
        g[ax] = fix;
        g[tang[0]] = s1;
        g[tang[1]] = s2;
        if (d == 2) g[2] = 1;
    };
    auto face_dims = [&](int f, int& n1, int& n2) {
        const int ax = f / 2, sh[3] = {a, b, c};
        int q = 0, dims[2] = {1, 1};
        for (int k = 0; k < d; ++k)
            if (k != ax) dims[q++] = sh[k];
        n1 = dims[0];
        n2 = dims[1];
    };
    const int nf = P.nf();
    size_t q = 0;
    if (which == RB_POINTS_POTENTIAL || which == RB_POINTS_SOURCE) {
        for (int i = 0; i < nl; ++i) {
            double h[3] = {0.0, 0.0, 0.0};
            for (int k = 0; k < d; ++k) h[k] = P.leaf_h[(size_t)d * i + k];
            const double* hp = which == RB_POINTS_POTENTIAL ? h : P.h_last;
            for (int gk = 1; gk <= c; ++gk)
                for (int gj = 1; gj <= b; ++gj)
                    for (int gi = 1; gi <= a; ++gi, ++q) coord(i, gi, gj, gk, hp, xyz + 3 * q);
        }
        return RB_OK;
    }
    if (which == RB_POINTS_BOUNDARY) {
        // the root's faces in turn; a face's points are its leaves' in leaf order (a merged face
        // is child1's part then child2's), each leaf's in the face's own order
        for (int f = 0; f < nf; ++f)
            for (int i = 0; i < nl; ++i) {
                if (!lf.isb[(size_t)nf * i + f]) continue;
                int n1, n2;
                face_dims(f, n1, n2);
                const int ax = f / 2;
                for (int s2 = 1; s2 <= n2; ++s2)
                    for (int s1 = 1; s1 <= n1; ++s1, ++q) {
                        int g[3];
                        face_grid(f, s1, s2, g);
                        double pt[3];
                        coord(i, g[0], g[1], g[2], P.h_last, pt);
                        // face-local coordinates as fd_make_bndry_vec leaves them (fd_module.f90:636-651):
                        // the tangential coordinates in natural order
                        int k = 0;
                        double loc[3] = {0.0, 0.0, 0.0};
                        for (int t2 = 0; t2 < d; ++t2)
                            if (t2 != ax) loc[k++] = pt[t2];
                        xyz[3 * q] = loc[0];
                        xyz[3 * q + 1] = loc[1];
                        xyz[3 * q + 2] = 0.0;
                    }
            }
        return RB_OK;
    }
    if (which == RB_POINTS_SOLUTION) {
        for (int i = 0; i < nl; ++i) {
            for (int f = 0; f < nf; ++f) {
                int n1, n2;
                face_dims(f, n1, n2);
                for (int s2 = 1; s2 <= n2; ++s2)
                    for (int s1 = 1; s1 <= n1; ++s1, ++q) {
                        int g[3];
                        face_grid(f, s1, s2, g);
                        coord(i, g[0], g[1], g[2], P.h_last, xyz + 3 * q);
                    }
            }
            for (int gk = 1; gk <= c; ++gk)
                for (int gj = 1; gj <= b; ++gj)
                    for (int gi = 1; gi <= a; ++gi, ++q) coord(i, gi, gj, gk, P.h_last, xyz + 3 * q);
        }
        return RB_OK;
    }
    return RB_ERR_INVALID;
}

// Enqueues the factor of t->d_k on the main stream: replayed as a graph, or launched directly
// with progress events (rec) for a solve that overlaps it (before_root_tail: see run_factor; the
// launches it makes are its own).
static int launch_factor(rb_tree* t, const std::vector<cudaEvent_t>* rec,
                         const std::function<int()>* before_root_tail = nullptr) {
    int rc;
    const long long l0 = launch_count();
    long long hook_launches = 0;
    t->factor_deferred = false;
    RB_CK(cudaEventRecord(t->ev[0], t->stream));
    if (rec) {
        std::function<int()> counted;
        if (before_root_tail)
            counted = [&] {
                const long long h0 = launch_count();
                const int r = (*before_root_tail)();
                hook_launches = launch_count() - h0;
                return r;
            };
        if ((rc = run_factor(t, t->d_k, rec, before_root_tail ? &counted : nullptr))) return rc;
    } else if ((rc = run_graphed(t, t->gx_factor, t->gx_factor_launches, t->factor_runs,
                                 [&] { return run_factor(t, t->d_k); }))) {
        return rc;
    }
    RB_CK(cudaMemcpyAsync(t->h_status, t->d_status, sizeof(int), cudaMemcpyDeviceToHost, t->stream));
    RB_CK(cudaEventRecord(t->ev[1], t->stream));
    t->factor_launches = launch_count() - l0 - hook_launches;
    t->factor_pending = true;
    return RB_OK;
}

// Waits for the last factor (launching it first if it was deferred), takes its time and its
// status (zero pivots) and reports them.
static int settle_factor(rb_tree* t) {
    if (t->factor_deferred) {
        if (int rc = launch_factor(t, nullptr)) return rc;
    }
    if (!t->factor_pending) return RB_OK;
    t->factor_pending = false;
    RB_CK(cudaEventSynchronize(t->ev[1]));
    float ms = 0.f;
    RB_CK(cudaEventElapsedTime(&ms, t->ev[0], t->ev[1]));
    t->f_time = ms * 1e-3;
    timers_collect(t);
    if (*t->h_status) {
        t->factored = false;
        t->nrhs = 0;
        if (*t->h_status & (RB_STATUS_GJ_TIMEOUT | RB_TC5_TIMEOUT))
            return fail(t, RB_ERR_CUDA, "a device wait timed out during the factorization");
        return fail(t, RB_ERR_NUMERIC, "zero pivot met while inverting a leaf or interface matrix");
    }
    if (t->verbose) std::printf("RTR computation completed.\nFactorization completed.\n");
    return RB_OK;
}

// Waits until the last solve's solution is in device memory and reports a failed factor.  After a
// solve that ran beside its factor the factor may still be finishing the root's own map, which no
// solve reads: its status word is complete once the root's interface inverse is, and the solve
// copied it then.
static int settle_solution(rb_tree* t) {
    if (!t->solve_overlapped) return settle_factor(t);
    RB_CK(cudaEventSynchronize(t->ev[3]));
    if (t->h_status[1]) {
        t->factored = false;
        t->nrhs = 0;
        return fail(t, RB_ERR_NUMERIC, "zero pivot met while inverting a leaf or interface matrix");
    }
    return RB_OK;
}

static int factor_common(rb_tree* t, const double* k, int precision, bool host, int sync) {
    if (!t) return RB_ERR_INVALID;
    if (!k) return fail(t, RB_ERR_INVALID, "rb_tree_factor: null potential samples");
    if (precision != RB_PREC_FP64 && precision != RB_PREC_MIXED)
        return fail(t, RB_ERR_INVALID, "precision mode " + std::to_string(precision) + " is not defined");
    if (precision == RB_PREC_MIXED && t->P.d != 2)
        return fail(t, RB_ERR_UNSUPPORTED, "the mixed-precision factorization is 2D only");
    int rc = ensure_factor_storage(t);
    if (rc) return rc;
    // a previous factor nobody waited for: report it, unless this call asks not to wait at all;
    // one that was deferred and never needed is dropped
    t->factor_deferred = false;
    if (!host && !sync) t->factor_pending = false;
    else if ((rc = settle_factor(t))) return rc;
    const Plan& P = t->P;
    const size_t nint = (size_t)P.nleaves() * P.leaf_interior();
    t->factored = false;
    t->nrhs = 0;
    if (precision != t->prec) {
        // the mixed factor launches other kernels on some levels: capture its own graph
        t->prec = precision;
        drop_graph(t->gx_factor);
        t->factor_runs = 0;
    }
    if (precision == RB_PREC_MIXED && (rc = ensure_mixed_factor_plan(t))) return rc;
    if (t->timing == 1) {
        timers_collect(t);
        t->stage_ms.clear();
    }
    for (auto& e : t->ev)
        if (!e) RB_CK(cudaEventCreate(&e));
    // the factor always reads the handle's own copy, so one captured graph serves every call.  A
    // host array is copied on the copy stream and waited for here, so that the caller may reuse
    // it as soon as this returns, even when the factor itself is still running.
    if (host) {
        RB_CK(cudaStreamWaitEvent(t->stream3, t->ev[1], 0));      // the last factor read d_k
        RB_CK(cudaMemcpyAsync(t->d_k, k, nint * sizeof(z), cudaMemcpyHostToDevice, t->stream3));
        RB_CK(cudaEventRecord(t->ev_copy, t->stream3));
        RB_CK(cudaStreamSynchronize(t->stream3));
        RB_CK(cudaStreamWaitEvent(t->stream, t->ev_copy, 0));
    } else {
        RB_CK(cudaMemcpyAsync(t->d_k, k, nint * sizeof(z), cudaMemcpyDeviceToDevice, t->stream));
    }
    t->factored = true;
    // RB_FLAG_ASYNC_FACTOR: nothing is launched yet; a solve that follows runs beside the factor
    if (t->async_factor && t->timing == 0 && (host || !sync)) {
        t->factor_deferred = true;
        return RB_OK;
    }
    if ((rc = launch_factor(t, nullptr))) return rc;
    if ((host && !t->async_factor) || (!host && sync)) return settle_factor(t);
    return RB_OK;
}

int rb_tree_factor(rb_tree* t, const double* k, int precision) { return factor_common(t, k, precision, true, 1); }
int rb_tree_factor_device(rb_tree* t, const double* dk, int precision, int sync) {
    return factor_common(t, dk, precision, false, sync);
}

static int solve_common(rb_tree* t, int nrhs, const double* f, const double* g, bool host, int sync) {
    if (!t) return RB_ERR_INVALID;
    if (!t->factored) return fail(t, RB_ERR_NOT_FACTORED, "Error: Robin Tree must be factored first.");
    if (nrhs <= 0) return fail(t, RB_ERR_INVALID, "rb_tree_solve: nrhs must be positive");
    if (!g) return fail(t, RB_ERR_INVALID, "rb_tree_solve: null boundary data");
    int rc = ensure_solve_storage(t, nrhs);
    if (rc) return rc;
    const Plan& P = t->P;
    const size_t nint = (size_t)P.nleaves() * P.leaf_interior();
    const size_t nroot = (size_t)P.lv[0].nb;
    const cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    t->nrhs = 0;
    t->solve_overlapped = false;
    if (t->prec == RB_PREC_MIXED) {
        // mixed precision: a host-steered refinement loop on the copy stream.  Inputs go up there
        // (beside a factor that may be running); with an asynchronous factor pending, the first
        // sweep waits for the factor level by level as in the FP64 overlap, and the corrections
        // follow it.  The root's Y1, Y2 and own map (read by no solve) may still run behind.
        const bool overlap = t->factor_deferred && t->timing == 0;
        cudaStream_t ss = overlap ? t->stream3 : t->stream;
        if (!overlap) {
            if (t->factor_deferred && (rc = launch_factor(t, nullptr))) return rc;
            if ((rc = settle_factor(t))) return rc;
        }
        RB_CK(cudaEventRecord(t->ev_copy, t->stream));          // device inputs are ordered there
        RB_CK(cudaStreamWaitEvent(ss, t->ev_copy, 0));
        RB_CK(cudaStreamWaitEvent(ss, t->ev[3], 0));            // the last read-back is done
        RB_CK(f ? cudaMemcpyAsync(t->d_f, f, nrhs * nint * sizeof(z), kind, ss)
                  : cudaMemsetAsync(t->d_f, 0, nrhs * nint * sizeof(z), ss));
        RB_CK(cudaMemcpyAsync(t->gbuf[0], g, nrhs * nroot * sizeof(z), kind, ss));
        RB_CK(cudaEventRecord(t->ev[2], ss));
        if (overlap && (rc = launch_factor(t, &t->ev_lvl))) return rc;
        const long long l0 = launch_count();
        rc = refine_solve(t, nrhs, ss, overlap ? &t->ev_lvl : nullptr);
        t->solve_launches = launch_count() - l0;
        if (overlap) {
            // every status write of the factor precedes the root level's event, which the first
            // sweep waited for
            RB_CK(cudaMemcpyAsync(t->h_status + 1, t->d_status, sizeof(int), cudaMemcpyDeviceToHost, ss));
        }
        RB_CK(cudaEventRecord(t->ev[3], ss));
        if (overlap) RB_CK(cudaStreamWaitEvent(t->stream, t->ev[3], 0));
        RB_CK(cudaStreamSynchronize(ss));
        if (overlap) {
            t->solve_overlapped = true;
            if (t->h_status[1]) {
                t->factored = false;
                t->nrhs = 0;
                return fail(t, (t->h_status[1] & RB_STATUS_ZERO_PIVOT) ? RB_ERR_NUMERIC : RB_ERR_CUDA,
                            "the factorization failed (zero pivot or a device wait timed out)");
            }
        }
        if (rc) return rc;
        float ms = 0.f;
        RB_CK(cudaEventElapsedTime(&ms, t->ev[2], t->ev[3]));
        t->s_time = ms * 1e-3;
        timers_collect(t);
        if (t->verbose) std::printf("Elliptic solve completed.\n");
        t->nrhs = nrhs;
        return RB_OK;
    }
    if (t->factor_deferred && t->timing == 0) {
        // factor and solve together: the factor on the main stream, the solve on the copy stream
        // right after its inputs, each solve level waiting for that level of the factor; the main
        // stream then waits for the solve, so later calls see both finished.  With host buffers
        // the caller reads the solution back next, so the solve is put first: the root's Y1, Y2
        // and own map (which no solve reads) wait for it and overlap the read-back instead of
        // competing with the solve's last levels.
        RB_CK(cudaEventRecord(t->ev_copy, t->stream));       // device inputs are ordered there
        RB_CK(cudaStreamWaitEvent(t->stream3, t->ev_copy, 0));
        RB_CK(f ? cudaMemcpyAsync(t->d_f, f, nrhs * nint * sizeof(z), kind, t->stream3)
                  : cudaMemsetAsync(t->d_f, 0, nrhs * nint * sizeof(z), t->stream3));
        RB_CK(cudaMemcpyAsync(t->gbuf[0], g, nrhs * nroot * sizeof(z), kind, t->stream3));
        const std::function<int()> enqueue_solve = [&]() -> int {
            const long long l0 = launch_count();
            RB_CK(cudaEventRecord(t->ev[2], t->stream3));
            if (int r = run_solve(t, nrhs, t->stream3, &t->ev_lvl)) return r;
            // every status write (leaf factor, interface inverses) precedes the root level's
            // event, which the solve waited for
            RB_CK(cudaMemcpyAsync(t->h_status + 1, t->d_status, sizeof(int), cudaMemcpyDeviceToHost, t->stream3));
            RB_CK(cudaEventRecord(t->ev[3], t->stream3));
            RB_CK(cudaStreamWaitEvent(t->stream, t->ev[3], 0));
            t->solve_launches = launch_count() - l0;
            return RB_OK;
        };
        if (host) {
            if ((rc = launch_factor(t, &t->ev_lvl, &enqueue_solve))) return rc;
        } else {
            if ((rc = launch_factor(t, &t->ev_lvl))) return rc;
            if ((rc = enqueue_solve())) return rc;
        }
        t->solve_overlapped = true;
    } else {
        if (t->factor_deferred && (rc = launch_factor(t, nullptr))) return rc;
        if (host) {
            // host right-hand sides go up on the copy stream, beside a factor that may still run on
            // the main stream; the copy waits until the last solve has read its buffers
            RB_CK(cudaStreamWaitEvent(t->stream3, t->ev[3], 0));
            RB_CK(f ? cudaMemcpyAsync(t->d_f, f, nrhs * nint * sizeof(z), kind, t->stream3)
                  : cudaMemsetAsync(t->d_f, 0, nrhs * nint * sizeof(z), t->stream3));
            RB_CK(cudaMemcpyAsync(t->gbuf[0], g, nrhs * nroot * sizeof(z), kind, t->stream3));
            RB_CK(cudaEventRecord(t->ev_copy, t->stream3));
            RB_CK(cudaStreamWaitEvent(t->stream, t->ev_copy, 0));
        } else {
            RB_CK(f ? cudaMemcpyAsync(t->d_f, f, nrhs * nint * sizeof(z), kind, t->stream)
                  : cudaMemsetAsync(t->d_f, 0, nrhs * nint * sizeof(z), t->stream));
            RB_CK(cudaMemcpyAsync(t->gbuf[0], g, nrhs * nroot * sizeof(z), kind, t->stream));
        }
        if ((rc = wait_readback(t, t->stream))) return rc;
        RB_CK(cudaEventRecord(t->ev[2], t->stream));
        const long long l0 = launch_count();
        if (t->gx_solve_rhs != nrhs) {     // the solve sequence depends on the RHS count
            drop_graph(t->gx_solve);
            t->gx_solve_rhs = nrhs;
            t->solve_runs = 0;
        }
        if ((rc = run_graphed(t, t->gx_solve, t->gx_solve_launches, t->solve_runs,
                              [&] { return run_solve(t, nrhs, t->stream); })))
            return rc;
        t->solve_launches = launch_count() - l0;
        RB_CK(cudaEventRecord(t->ev[3], t->stream));
    }
    if (host || sync) {
        if (t->solve_overlapped) {
            if ((rc = settle_solution(t))) return rc;
        } else {
            RB_CK(cudaStreamSynchronize(t->stream));
            if ((rc = settle_factor(t))) return rc;
        }
        float ms = 0.f;       // beside an overlapped factor this spans the wait for its levels too
        RB_CK(cudaEventElapsedTime(&ms, t->ev[2], t->ev[3]));
        t->s_time = ms * 1e-3;
        timers_collect(t);
        if (t->verbose) std::printf("Elliptic solve completed.\n");
    }
    t->nrhs = nrhs;
    return RB_OK;
}

int rb_tree_solve(rb_tree* t, int nrhs, const double* f, const double* g) {
    return solve_common(t, nrhs, f, g, true, 1);
}
int rb_tree_solve_device(rb_tree* t, int nrhs, const double* f, const double* g, int sync) {
    return solve_common(t, nrhs, f, g, false, sync);
}

int rb_get_solution(const rb_tree* tc, int irhs, double* u, double* boxes) {
    rb_tree* t = const_cast<rb_tree*>(tc);
    if (!t || !u) return RB_ERR_INVALID;
    if (int rc = (t->factor_deferred || t->nrhs == 0) ? settle_factor(t) : settle_solution(t)) return rc;
    if (!t->factored) return fail(t, RB_ERR_NOT_FACTORED, "Error in GET_SOLUTION: Robin Tree not factored.");
    if (irhs < 0 || irhs >= t->nrhs) return fail(t, RB_ERR_NO_SOLUTION, "get_solution: no solution for this right-hand side");
    const Plan& P = t->P;
    const size_t per = (size_t)P.nleaves() * P.leaf_n();
    // on the copy stream after the solve: a factor's remaining root work may run beside it
    RB_CK(cudaStreamWaitEvent(t->stream3, t->ev[3], 0));
    RB_CK(cudaMemcpyAsync(u, t->sol + (size_t)irhs * per, per * sizeof(z), cudaMemcpyDeviceToHost, t->stream3));
    RB_CK(cudaStreamSynchronize(t->stream3));
    if (boxes) {
        const PlanLevel& lf = P.lv[P.L];
        for (int i = 0; i < lf.nnodes; ++i)
            for (int j = 0; j < 3; ++j) {
                boxes[6 * i + 2 * j] = lf.lo[3 * i + j];
                boxes[6 * i + 2 * j + 1] = lf.hi[3 * i + j];
            }
    }
    return RB_OK;
}

int rb_get_solution_async(const rb_tree* tc, int irhs, double* u, double* boxes) {
    rb_tree* t = const_cast<rb_tree*>(tc);
    if (!t || !u) return RB_ERR_INVALID;
    if (int rc = (t->factor_deferred || t->nrhs == 0) ? settle_factor(t) : settle_solution(t)) return rc;
    if (!t->factored) return fail(t, RB_ERR_NOT_FACTORED, "Error in GET_SOLUTION: Robin Tree not factored.");
    if (irhs < 0 || irhs >= t->nrhs) return fail(t, RB_ERR_NO_SOLUTION, "get_solution: no solution for this right-hand side");
    if (!t->stream5) {
        int lo = 0, hi = 0;
        RB_CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        RB_CK(cudaStreamCreateWithPriority(&t->stream5, cudaStreamNonBlocking, lo));
    }
    if (!t->ev_d2h) RB_CK(cudaEventCreateWithFlags(&t->ev_d2h, cudaEventDisableTiming));
    const Plan& P = t->P;
    const size_t per = (size_t)P.nleaves() * P.leaf_n();
    RB_CK(cudaStreamWaitEvent(t->stream5, t->ev[3], 0));        // the solve that wrote the solution
    RB_CK(cudaMemcpyAsync(u, t->sol + (size_t)irhs * per, per * sizeof(z), cudaMemcpyDeviceToHost, t->stream5));
    RB_CK(cudaEventRecord(t->ev_d2h, t->stream5));
    t->d2h_pending = true;
    if (boxes) {
        const PlanLevel& lf = P.lv[P.L];
        for (int i = 0; i < lf.nnodes; ++i)
            for (int j = 0; j < 3; ++j) {
                boxes[6 * i + 2 * j] = lf.lo[3 * i + j];
                boxes[6 * i + 2 * j + 1] = lf.hi[3 * i + j];
            }
    }
    return RB_OK;
}

int rb_tree_sync(const rb_tree* tc) {
    rb_tree* t = const_cast<rb_tree*>(tc);
    if (!t) return RB_ERR_INVALID;
    if (t->stream5) RB_CK(cudaStreamSynchronize(t->stream5));
    return RB_OK;
}

int rb_get_solution_device(const rb_tree* tc, double* du, int sync) {
    rb_tree* t = const_cast<rb_tree*>(tc);
    if (!t || !du) return RB_ERR_INVALID;
    if (!t->factored) return fail(t, RB_ERR_NOT_FACTORED, "Error in GET_SOLUTION: Robin Tree not factored.");
    if (t->nrhs <= 0) return fail(t, RB_ERR_NO_SOLUTION, "get_solution: no solve has run");
    const Plan& P = t->P;
    const size_t tot = (size_t)t->nrhs * P.nleaves() * P.leaf_n();
    RB_CK(cudaMemcpyAsync(du, t->sol, tot * sizeof(z), cudaMemcpyDeviceToDevice, t->stream));
    if (sync) RB_CK(cudaStreamSynchronize(t->stream));
    return RB_OK;
}

int rb_tree_times(const rb_tree* tc, double* f_time, double* s_time) {
    rb_tree* t = const_cast<rb_tree*>(tc);
    if (!t) return RB_ERR_INVALID;
    if (int rc = settle_factor(t)) return rc;
    if (f_time) *f_time = t->f_time;
    if (s_time) *s_time = t->s_time;
    return RB_OK;
}

void* rb_tree_stream(const rb_tree* t) { return t ? (void*)t->stream : nullptr; }

int rb_tree_set_timing(rb_tree* t, int mode) {
    if (!t || mode < 0 || mode > 2) return RB_ERR_INVALID;
    t->timing = mode;
    return RB_OK;
}

int rb_tree_stage_times(const rb_tree* tc, double* ms, double* flops, const char** names, int n) {
    rb_tree* t = const_cast<rb_tree*>(tc);
    if (!t) return RB_ERR_INVALID;
    if (!t->timers.empty()) {      // entries of asynchronous calls: wait for them
        if (t->stream) RB_CK(cudaStreamSynchronize(t->stream));
        timers_collect(t);
    }
    const int cnt = (int)t->stage_ms.size();
    for (int i = 0; i < std::min(n, cnt); ++i) {
        if (ms) ms[i] = t->stage_ms[i].ms;
        if (flops) flops[i] = t->stage_ms[i].flops;
        if (names) names[i] = t->stage_ms[i].name.c_str();
    }
    return cnt;
}

int rb_tree_clear_stage_times(rb_tree* t) {
    if (!t) return RB_ERR_INVALID;
    if (t->stream) RB_CK(cudaStreamSynchronize(t->stream));
    timers_collect(t);
    t->stage_ms.clear();
    return RB_OK;
}

int rb_tree_level_shape(const rb_tree* t, int level, int32_t* shape) {
    if (!t || !shape || level < 0 || level > t->P.L) return RB_ERR_INVALID;
    shape[0] = t->P.lv[level].nnodes;
    shape[1] = t->P.lv[level].a;
    shape[2] = t->P.lv[level].b;
    shape[3] = t->P.lv[level].c;
    return RB_OK;
}

int rb_tree_get_rtr(const rb_tree* tc, int level, int node, double* out) {
    rb_tree* t = const_cast<rb_tree*>(tc);
    if (!t || !out) return RB_ERR_INVALID;
    if (int rc = settle_factor(t)) return rc;
    if (!t->factored) return fail(t, RB_ERR_NOT_FACTORED, "Error: Robin Tree must be factored first.");
    const Plan& P = t->P;
    if (level < 0 || level > P.L || node < 0 || node >= P.lv[level].nnodes)
        return fail(t, RB_ERR_INVALID, "rb_tree_get_rtr: level or node out of range");
    const int nb = P.lv[level].nb;
    const z* src = nullptr;
    if (level == P.L) src = t->leaf_Y + (long long)node * nb * P.leaf_n();
    else if (t->rtr[level]) src = t->rtr[level] + (long long)node * nb * nb;
    if (!src) return fail(t, RB_ERR_INVALID, "rb_tree_get_rtr: the root RtR was not formed (RB_FLAG_SKIP_ROOT_RTR)");
    RB_CK(cudaMemcpyAsync(out, src, (size_t)nb * nb * sizeof(z), cudaMemcpyDeviceToHost, t->stream));
    RB_CK(cudaStreamSynchronize(t->stream));
    return RB_OK;
}

int rb_tree_set_refinement(rb_tree* t, double tol, int max_iter) {
    if (!t) return RB_ERR_INVALID;
    if (!(tol > 0.0) || !(tol < 1.0) || max_iter < 1 || max_iter > 100)
        return fail(t, RB_ERR_INVALID, "rb_tree_set_refinement: tol must be in (0, 1) and max_iter in 1..100");
    t->refine_tol = tol;
    t->refine_maxit = max_iter;
    return RB_OK;
}

int rb_tree_refine_info(const rb_tree* t, int32_t* iters, double* contraction, double* est_err, double* residual) {
    if (!t) return RB_ERR_INVALID;
    if (iters) *iters = t->refine_iters;
    if (contraction) *contraction = t->refine_rho;
    if (est_err) *est_err = t->refine_est;
    if (residual) *residual = t->refine_res;
    return RB_OK;
}

int rb_tree_launch_counts(const rb_tree* t, int64_t* fl, int64_t* sl) {
    if (!t) return RB_ERR_INVALID;
    if (fl) *fl = t->factor_launches;
    if (sl) *sl = t->solve_launches;
    return RB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------
// Accessors for the serving loop (rb_server.cpp), which drives handles through the C-ABI.

namespace rb {
// storage and launch batches of an FP64 factorization (for a forest that runs the factor itself)
int tree_prepare_factor(rb_tree* t) {
    if (int rc = settle_factor(t)) return rc;
    t->factor_deferred = false;
    return ensure_factor_storage(t);
}
// a factorization that a forest completed on the tree's storage
void tree_mark_factored(rb_tree* t, double f_time) {
    t->factored = true;
    t->factor_pending = false;
    t->factor_deferred = false;
    t->nrhs = 0;
    if (t->prec != RB_PREC_FP64) {
        t->prec = RB_PREC_FP64;
        drop_graph(t->gx_factor);
        t->factor_runs = 0;
    }
    t->f_time = f_time;
}
// device address of the solutions of the last solve, [rhs][leaf][leaf_n]
const z* tree_solutions(const rb_tree* t) { return t->sol; }
int tree_device(const rb_tree* t) { return t->device; }
// bytes a factorization plus the buffers of one solve of nrhs right-hand sides take on the device
// (persistent factor storage as rb_tree_create's budget check counts it, the solve's per-level
// vectors, its split-K workspace bound and, for a mixed-precision factor, the refinement buffers)
double tree_bytes_estimate(const rb_tree* t, int nrhs, int precision) {
    const Plan& Q = t->P;
    const double ab = (double)Q.leaf_interior();
    double need = leaf_factor_bytes(Q);
    double per_rhs = (double)Q.nleaves() * (ab + Q.leaf_n()) * 16.0;
    for (int l = 0; l < Q.L; ++l) {
        need += (double)Q.lv[l].nnodes *
                ((double)Q.lv[l].nb * Q.lv[l].nb + (t->kform ? 3.0 : 2.0) * Q.lv[l].m * Q.lv[l].m +
                 2.0 * Q.lv[l].m * (Q.lv[l].n1 + Q.lv[l].n2)) * 16.0;
        per_rhs += 2.0 * Q.lv[l].nnodes * Q.lv[l].nb * 16.0;
    }
    per_rhs *= 1.5;                                   // split-K workspace and the root's x1, x2
    if (precision == RB_PREC_MIXED) per_rhs += (double)Q.nleaves() * (Q.leaf_n() + Q.leaf_nb()) * 16.0;
    return need * 1.02 + per_rhs * nrhs + (64 << 20);
}
}  // namespace rb

// ---------------------------------------------------------------------------------------------------
// Device-side sampling, check_solution, save / load.

static int ensure_points(rb_tree* t, int which, double** out) {
    const int idx = which == RB_POINTS_POTENTIAL ? 0 : which == RB_POINTS_SOURCE ? 1 : 2;
    if (!t->d_pts[idx]) {
        const Plan& P = t->P;
        const size_t n = which == RB_POINTS_BOUNDARY ? (size_t)P.lv[0].nb
                                                     : (size_t)P.nleaves() * P.leaf_interior();
        std::vector<double> h(3 * n);
        int rc = rb_tree_sample_points(t, which, h.data());
        if (rc) return rc;
        if ((rc = alloc_n(t, t->bufs, 3 * n, &t->d_pts[idx]))) return rc;
        RB_CK(cudaMemcpy(t->d_pts[idx], h.data(), 3 * n * sizeof(double), cudaMemcpyHostToDevice));
    }
    *out = t->d_pts[idx];
    return RB_OK;
}

static int upload_params(rb_tree* t, const double* par, size_t n) {
    if (n > t->par_cap) {
        int rc = alloc_n(t, t->bufs, n, &t->d_par);
        if (rc) return rc;
        t->par_cap = n;
    }
    if (n) RB_CK(cudaMemcpyAsync(t->d_par, par, n * sizeof(double), cudaMemcpyHostToDevice, t->stream));
    return RB_OK;
}

int rb_tree_sample_device(rb_tree* t, int kind, int count, const double* params, double* d_f, double* d_g,
                          int sync) {
    if (!t || !params || count < 0) return RB_ERR_INVALID;
    if (t->P.d != 2) return fail(t, RB_ERR_UNSUPPORTED, "device sampling is 2D only");
    int rc;
    if (!t->stream) RB_CK(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking));
    const Plan& P = t->P;
    const long long nint = (long long)P.nleaves() * P.leaf_interior();
    const int nb = P.lv[0].nb;
    cudaStream_t s = t->stream;
    double* pts = nullptr;
    if (kind == RB_FIELD_BUMP_POTENTIAL) {
        if (!d_f) return fail(t, RB_ERR_INVALID, "rb_tree_sample_device: the potential needs d_f");
        if ((rc = ensure_points(t, RB_POINTS_POTENTIAL, &pts))) return rc;
        if ((rc = upload_params(t, params + 3, 3 * (size_t)count))) return rc;
        RB_LAUNCH(sample_bump(pts, nint, params[0], params[1], params[2], count, t->d_par, (z*)d_f, s));
    } else if (kind == RB_FIELD_POINT_SOURCE) {
        if ((rc = ensure_points(t, RB_POINTS_SOURCE, &pts))) return rc;
        if ((rc = upload_params(t, params, 3 * (size_t)count))) return rc;
        if (d_f) RB_LAUNCH(sample_point_sources(pts, nint, count, t->d_par, (z*)d_f, s));
        if (d_g) RB_CK(cudaMemsetAsync(d_g, 0, (size_t)count * nb * sizeof(z), s));
    } else if (kind == RB_FIELD_PLANE_WAVE) {
        if ((rc = ensure_points(t, RB_POINTS_BOUNDARY, &pts))) return rc;
        if ((rc = upload_params(t, params, 3 * (size_t)count))) return rc;
        const double dom4[4] = {t->geom.domain[0], t->geom.domain[1], t->geom.domain[2], t->geom.domain[3]};
        if (d_g) RB_LAUNCH(sample_plane_waves(pts, nb, P.lv[0].a, P.lv[0].b, dom4, count, t->d_par, (z*)d_g, s));
        if (d_f) RB_CK(cudaMemsetAsync(d_f, 0, (size_t)count * nint * sizeof(z), s));
    } else {
        return fail(t, RB_ERR_INVALID, "rb_tree_sample_device: unknown kind " + std::to_string(kind));
    }
    if (sync) RB_CK(cudaStreamSynchronize(s));
    return RB_OK;
}

static int check_common(rb_tree* t, int irhs, const double* uex, bool host, int norm, int rel, double* err) {
    if (!t || !uex || !err) return RB_ERR_INVALID;
    int rc;
    if ((rc = settle_factor(t))) return rc;
    if (!t->factored) return fail(t, RB_ERR_NOT_FACTORED, "Error in GET_SOLUTION: Robin Tree not factored.");
    if (irhs < 0 || irhs >= t->nrhs)
        return fail(t, RB_ERR_NO_SOLUTION, "check_solution: no solution for this right-hand side");
    const Plan& P = t->P;
    const int nl = P.nleaves(), n = P.leaf_n();
    const size_t per = (size_t)nl * n;
    if (!t->d_err && (rc = alloc_n(t, t->bufs, (size_t)nl, &t->d_err))) return rc;
    const z* ue = reinterpret_cast<const z*>(uex);
    if (host) {
        if (!t->d_uex && (rc = alloc_n(t, t->bufs, per, &t->d_uex))) return rc;
        RB_CK(cudaMemcpyAsync(t->d_uex, uex, per * sizeof(z), cudaMemcpyHostToDevice, t->stream));
        ue = t->d_uex;
    }
    RB_LAUNCH(check_solution(t->sol + (size_t)irhs * per, ue, nl, n, norm, rel, t->d_err, t->stream));
    RB_CK(cudaMemcpyAsync(err, t->d_err, nl * sizeof(double), cudaMemcpyDeviceToHost, t->stream));
    RB_CK(cudaStreamSynchronize(t->stream));
    return RB_OK;
}

int rb_check_solution(const rb_tree* t, int irhs, const double* u_exact, int norm, int rel, double* err) {
    return check_common(const_cast<rb_tree*>(t), irhs, u_exact, true, norm, rel, err);
}
int rb_check_solution_device(const rb_tree* t, int irhs, const double* d_u_exact, int norm, int rel, double* err) {
    return check_common(const_cast<rb_tree*>(t), irhs, d_u_exact, false, norm, rel, err);
}

// Every buffer the solve reads after a factorization, in file order.
static std::vector<std::pair<z*, size_t>> factor_sections(rb_tree* t) {
    const Plan& P = t->P;
    const size_t nl = P.nleaves(), a = P.leaf_a(), b = P.leaf_b(), nb = P.leaf_nb(), n = P.leaf_n();
    std::vector<std::pair<z*, size_t>> v;
    v.push_back({t->leaf_sinv, P.d == 2 ? nl * b * a * a : nl * n * n});   // 3D: the dense leaf inverses
    v.push_back({t->leaf_Y, nl * nb * n});
    for (int l = 0; l < P.L; ++l) {
        const PlanLevel& p = P.lv[l];
        const size_t mm = (size_t)p.nnodes * p.m * p.m;
        if (t->rtr[l]) v.push_back({t->rtr[l], (size_t)p.nnodes * p.nb * p.nb});
        v.push_back({t->dinv[l], mm});
        v.push_back({t->sinv[l], mm});
        if (t->kform) v.push_back({t->kinv[l], mm});
        if (l > 0) {
            const size_t ny = (size_t)p.nnodes * p.m * (p.n1 + p.n2);
            v.push_back({t->Y1[l], ny});
            v.push_back({t->Y2[l], ny});
        }
    }
    return v;
}

struct SaveHeader {
    char magic[8];
    uint32_t version;
    uint32_t geom_bytes;
    rb_geom geom;
    int32_t kform;
    int32_t nsections;
};
static const char kMagic[8] = {'R', 'B', 'T', 'R', 'E', 'E', 'F', '1'};
// 2: [Y1; Y2] of every level below the root follow each level's inverses
static const uint32_t kSaveVersion = 2;

int rb_tree_save(const rb_tree* tc, const char* path) {
    rb_tree* t = const_cast<rb_tree*>(tc);
    if (!t || !path) return RB_ERR_INVALID;
    int rc;
    if ((rc = settle_factor(t))) return rc;
    if (!t->factored) return fail(t, RB_ERR_NOT_FACTORED, "Error: Robin Tree must be factored first.");
    RB_CK(cudaStreamSynchronize(t->stream));
    const auto secs = factor_sections(t);
    SaveHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = kSaveVersion;
    h.geom_bytes = sizeof(rb_geom);
    h.geom = t->geom;
    h.kform = t->kform ? 1 : 0;
    h.nsections = (int32_t)secs.size();
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(t, RB_ERR_INVALID, std::string("rb_tree_save: cannot open ") + path);
    bool ok = std::fwrite(&h, sizeof(h), 1, fp) == 1;
    std::vector<z> stage(std::min<size_t>(1 << 22, std::max<size_t>(1, secs.empty() ? 1 : secs[0].second)));
    for (const auto& sec : secs) {
        const uint64_t cnt = sec.second;
        ok = ok && std::fwrite(&cnt, sizeof(cnt), 1, fp) == 1;
        for (size_t off = 0; ok && off < sec.second; off += stage.size()) {
            const size_t c = std::min(stage.size(), sec.second - off);
            if (cudaMemcpy(stage.data(), sec.first + off, c * sizeof(z), cudaMemcpyDeviceToHost) != cudaSuccess) {
                std::fclose(fp);
                return fail(t, RB_ERR_CUDA, "rb_tree_save: device read failed");
            }
            ok = std::fwrite(stage.data(), sizeof(z), c, fp) == c;
        }
    }
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return fail(t, RB_ERR_INVALID, std::string("rb_tree_save: write to ") + path + " failed");
    return RB_OK;
}

int rb_tree_load(const char* path, rb_tree** out) {
    if (!path || !out) return RB_ERR_INVALID;
    *out = nullptr;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) {
        g_create_error = std::string("rb_tree_load: cannot open ") + path;
        return RB_ERR_INVALID;
    }
    SaveHeader h{};
    if (std::fread(&h, sizeof(h), 1, fp) != 1 || std::memcmp(h.magic, kMagic, 8) != 0 || h.version != kSaveVersion ||
        h.geom_bytes != sizeof(rb_geom)) {
        std::fclose(fp);
        g_create_error = std::string("rb_tree_load: ") + path + " is not a factorized tree of this library";
        return RB_ERR_INVALID;
    }
    rb_tree* t = nullptr;
    int rc = rb_tree_create(&h.geom, &t);
    if (rc) {
        std::fclose(fp);
        return rc;
    }
    auto bail = [&](int code, const std::string& msg) {
        std::fclose(fp);
        g_create_error = msg;
        rb_tree_destroy(t);
        return code;
    };
    if ((int)t->kform != h.kform) return bail(RB_ERR_INVALID, "rb_tree_load: interface form differs from the file's");
    if ((rc = ensure_factor_storage(t))) return bail(rc, t->err);
    const auto secs = factor_sections(t);
    if ((int)secs.size() != h.nsections) return bail(RB_ERR_INVALID, "rb_tree_load: section count mismatch");
    std::vector<z> stage(std::min<size_t>(1 << 22, std::max<size_t>(1, secs.empty() ? 1 : secs[0].second)));
    for (const auto& sec : secs) {
        uint64_t cnt = 0;
        if (std::fread(&cnt, sizeof(cnt), 1, fp) != 1 || cnt != sec.second)
            return bail(RB_ERR_INVALID, "rb_tree_load: section size mismatch (file truncated or of another tree)");
        for (size_t off = 0; off < sec.second; off += stage.size()) {
            const size_t c = std::min(stage.size(), sec.second - off);
            if (std::fread(stage.data(), sizeof(z), c, fp) != c)
                return bail(RB_ERR_INVALID, "rb_tree_load: file truncated");
            if (cudaMemcpy(sec.first + off, stage.data(), c * sizeof(z), cudaMemcpyHostToDevice) != cudaSuccess)
                return bail(RB_ERR_CUDA, "rb_tree_load: device write failed");
        }
    }
    std::fclose(fp);
    t->factored = true;
    t->factor_pending = false;
    t->factor_deferred = false;
    *out = t;
    return RB_OK;
}
