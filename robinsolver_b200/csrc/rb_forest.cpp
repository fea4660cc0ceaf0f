// rb_forest.cpp -- several independent trees factored in one level-synchronous schedule, with a
// project autotuner for the GEMM tile shapes (include/robin_b200.h, rb_forest_*).
//
// The reference factors one tree by a serial recursion (compute_RTR, robin_tree_module.f90:375-401).
// A forest factors many trees of different sizes at once.  Trees are aligned by height above
// their leaves: at height h every tree with L >= h merges its level L - h.  Per height the whole
// forest runs
//   one batched launch forming A2, A1, K of every node of every tree (merge_form_kform_batch),
//   one launch per merge GEMM stage over the concatenated descriptors of all trees
//     (B1 = -A2 T1_iN, K -= A2 A1, Y1, Y2, parent map; uneven m, n, k in one launch),
//   one resident Gauss-Jordan launch per distinct interface size (at most two per height for
//     the serving/batching sets: interface sizes depend only on the leaf size and the height),
// so a forest of 64 trees takes about the launches of ONE tree.  The leaf stage runs each tree's
// leaf kernel on one of several streams.  The whole schedule is captured once into a CUDA graph
// and replayed.
//
// Autotuner: the first factor of a forest (with tuning on) times every applicable FP64 tile shape
// (DFMA 32x32, 64x64, 128x64; DMMA 32x32, 64x64, contiguous-k 64x64) on each concatenated GEMM
// stage with CUDA events, in a throw-away pass over the real data, and keeps the fastest per stage;
// the choices are cached process-wide by the stage's shape (count, max m, n, k, contiguity) so later
// forests of the same shapes skip the search.  Then the real factor runs with the chosen shapes.
// Every tile shape accumulates in FP64; the results agree with the one-tree factor to rounding.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "rb_tree_impl.hpp"

namespace rb {
int tree_prepare_factor(rb_tree* t);
void tree_mark_factored(rb_tree* t, double f_time);
}  // namespace rb

namespace {

struct GJGroup {
    int m = 0;
    int count = 0;
    GJDesc* d_desc = nullptr;
    z* flags = nullptr;
};

struct HeightPlan {
    int nforms = 0, max_m = 0;
    MergeFormDesc* d_forms = nullptr;
    GemmBatch K, M1, M2, M3, M4;
    std::vector<GJGroup> gj;
};

using Sig = std::tuple<int, int, int, int, bool>;
std::mutex g_tune_mu;
std::map<Sig, int> g_tuned;           // stage shape -> engine, process-wide

Sig sig_of(const GemmBatch& b) { return Sig(b.count, b.max_m, b.max_n, b.max_k, b.kcontig); }

}  // namespace

struct rb_forest {
    std::vector<rb_tree*> trees;
    int device = 0;
    int maxL = 0;
    cudaStream_t stream = nullptr;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> ev_fork, ev_join;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<HeightPlan> H;        // index = height 1..maxL
    int* d_status = nullptr;
    int* h_status = nullptr;
    std::vector<void*> bufs;
    cudaGraphExec_t gx = nullptr;
    int runs = 0;
    bool tuned = false;
    double f_time = 0.0;
    long long launches = 0;
    std::string err;
    // per-stage autotuning record (height, stage, engine, ms)
    struct TuneRec { int h; int stage; int engine; float ms; };
    std::vector<TuneRec> tune_log;
};

namespace {

#define FCK(call)                                                                                \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            f->err = std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call;        \
            return RB_ERR_CUDA;                                                                  \
        }                                                                                        \
    } while (0)

int falloc(rb_forest* f, size_t bytes, void** out) {
    *out = nullptr;
    if (bytes == 0) return RB_OK;
    cudaError_t e = cudaMalloc(out, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        f->err = std::string("cudaMalloc failed: ") + cudaGetErrorString(e);
        return RB_ERR_OUT_OF_MEMORY;
    }
    f->bufs.push_back(*out);
    return RB_OK;
}

// concatenation of the trees' descriptor arrays of one stage (device to device)
int concat_batches(rb_forest* f, const std::vector<const GemmBatch*>& parts, GemmBatch& out) {
    out = GemmBatch();
    int count = 0;
    for (const GemmBatch* b : parts) count += b->count;
    if (count == 0) return RB_OK;
    void* p = nullptr;
    if (int rc = falloc(f, sizeof(GemmDesc) * count, &p)) return rc;
    out.d_desc = static_cast<GemmDesc*>(p);
    out.kcontig = true;
    int off = 0;
    for (const GemmBatch* b : parts) {
        if (b->count == 0) continue;
        FCK(cudaMemcpy(out.d_desc + off, b->d_desc, sizeof(GemmDesc) * b->count, cudaMemcpyDeviceToDevice));
        off += b->count;
        out.max_m = std::max(out.max_m, b->max_m);
        out.max_n = std::max(out.max_n, b->max_n);
        out.max_k = std::max(out.max_k, b->max_k);
        out.flops += b->flops;
        out.kcontig = out.kcontig && b->kcontig;
    }
    out.count = count;
    return RB_OK;
}

int build_plan(rb_forest* f) {
    f->H.assign(f->maxL + 1, HeightPlan());
    for (int h = 1; h <= f->maxL; ++h) {
        HeightPlan& hp = f->H[h];
        std::vector<MergeFormDesc> forms;
        std::vector<const GemmBatch*> K, M1, M2, M3, M4;
        std::map<int, std::vector<GJDesc>> gj;
        for (rb_tree* t : f->trees) {
            const Plan& P = t->P;
            if (P.L < h) continue;
            const int l = P.L - h;
            const PlanLevel& p = P.lv[l];
            // the children's storage: leaf Y (first nb columns = RtR) or the level's RtR maps
            const z* rtr;
            long long stride, ld;
            if (l + 1 == P.L) {
                rtr = t->leaf_Y;
                stride = (long long)P.leaf_nb() * P.leaf_n();
                ld = P.leaf_nb();
            } else {
                rtr = t->rtr[l + 1];
                stride = (long long)P.lv[l + 1].nb * P.lv[l + 1].nb;
                ld = P.lv[l + 1].nb;
            }
            const int m = p.m;
            for (int i = 0; i < p.nnodes; ++i) {
                MergeFormDesc d{};
                d.t1 = rtr + (2LL * i) * stride;
                d.t2 = rtr + (2LL * i + 1) * stride;
                d.ld = ld;
                d.m = m;
                d.o1 = p.o1;
                d.o2 = p.o2;
                d.zeta = t->zeta;
                d.nu2 = zmul(t->nu, t->nu);
                d.a2 = t->dinv[l] + (long long)i * m * m;
                d.a1 = t->sinv[l] + (long long)i * m * m;
                d.k = t->kinv[l] + (long long)i * m * m;
                forms.push_back(d);
                GJDesc g{};
                g.A = t->kinv[l] + (long long)i * m * m;
                g.ld = m;
                g.ipiv = t->gj_ipiv + (long long)i * m;
                g.Zb = nullptr;        // set below: the group's own flag words, contiguous
                gj[m].push_back(g);
            }
            hp.max_m = std::max(hp.max_m, m);
            K.push_back(&t->fK[l]);
            M1.push_back(&t->fM1[l]);
            M2.push_back(&t->fM2[l]);
            M3.push_back(&t->fM3[l]);
            M4.push_back(&t->fM4[l]);
        }
        hp.nforms = (int)forms.size();
        if (hp.nforms > 65535) {
            f->err = "rb_forest: more than 65535 merges at one height";
            return RB_ERR_INVALID;
        }
        void* p = nullptr;
        if (int rc = falloc(f, sizeof(MergeFormDesc) * forms.size(), &p)) return rc;
        hp.d_forms = static_cast<MergeFormDesc*>(p);
        FCK(cudaMemcpy(hp.d_forms, forms.data(), sizeof(MergeFormDesc) * forms.size(), cudaMemcpyHostToDevice));
        if (int rc = concat_batches(f, K, hp.K)) return rc;
        if (int rc = concat_batches(f, M1, hp.M1)) return rc;
        if (int rc = concat_batches(f, M2, hp.M2)) return rc;
        if (int rc = concat_batches(f, M3, hp.M3)) return rc;
        if (int rc = concat_batches(f, M4, hp.M4)) return rc;
        for (auto& kv : gj) {
            GJGroup g;
            g.m = kv.first;
            g.count = (int)kv.second.size();
            const long long ws = gj_workspace_elems(g.m);
            if (int rc = falloc(f, sizeof(z) * std::max<long long>(1, ws * g.count), &p)) return rc;
            g.flags = static_cast<z*>(p);
            for (int i = 0; i < g.count; ++i) kv.second[i].Zb = g.flags + ws * i;
            if (int rc = falloc(f, sizeof(GJDesc) * g.count, &p)) return rc;
            g.d_desc = static_cast<GJDesc*>(p);
            FCK(cudaMemcpy(g.d_desc, kv.second.data(), sizeof(GJDesc) * g.count, cudaMemcpyHostToDevice));
            hp.gj.push_back(g);
        }
    }
    return RB_OK;
}

// one GEMM stage; with `tune`, every candidate engine is timed on it first (the results of the
// tuning pass are discarded by the real pass that follows)
int run_gemm(rb_forest* f, GemmBatch& b, int h, int stage, bool tune, cudaStream_t s) {
    if (b.count == 0) return RB_OK;
    if (tune) {
        int cand[8];
        const int nc = gemm_engine_candidates(b, cand);
        float best = 1e30f;
        int pick = -1;
        for (int c = 0; c < nc; ++c) {
            b.engine = cand[c];
            // a tile shape that cannot launch on this batch (its launch is refused before any
            // device work) is no candidate
            if (launch_gemm_batch(b, s) != cudaSuccess) {  // warm (and the first timing's cold start)
                cudaGetLastError();
                f->tune_log.push_back({h, stage, cand[c], -1.0f});
                continue;
            }
            FCK(cudaEventRecord(f->ev0, s));
            FCK(launch_gemm_batch(b, s));
            FCK(cudaEventRecord(f->ev1, s));
            FCK(cudaEventSynchronize(f->ev1));
            float ms = 0.f;
            FCK(cudaEventElapsedTime(&ms, f->ev0, f->ev1));
            f->tune_log.push_back({h, stage, cand[c], ms});
            if (ms < best) {
                best = ms;
                pick = cand[c];
            }
        }
        if (pick < 0) {
            f->err = "rb_forest: no GEMM tile shape could run a merge stage";
            return RB_ERR_CUDA;
        }
        b.engine = pick;
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[sig_of(b)] = pick;
    }
    FCK(launch_gemm_batch(b, s));
    return RB_OK;
}

int run_schedule(rb_forest* f, bool tune) {
    cudaStream_t s = f->stream;
    FCK(cudaMemsetAsync(f->d_status, 0, sizeof(int), s));
    // leaves: each tree's leaf kernel on a side stream
    FCK(cudaEventRecord(f->ev_fork[0], s));
    for (size_t i = 0; i < f->trees.size(); ++i) {
        rb_tree* t = f->trees[i];
        const Plan& P = t->P;
        cudaStream_t ss = f->side[i % f->side.size()];
        if (i < f->side.size()) FCK(cudaStreamWaitEvent(ss, f->ev_fork[0], 0));
        LeafGeom lg{P.leaf_a(), P.leaf_b(), P.leaf_nb(), P.leaf_n(), P.kb};
        FCK(leaf_block_factor(lg, P.nleaves(), t->d_h, t->d_k, t->leaf_sinv, t->leaf_Y, f->d_status, ss));
    }
    for (size_t j = 0; j < f->side.size() && j < f->trees.size(); ++j) {
        FCK(cudaEventRecord(f->ev_join[j], f->side[j]));
        FCK(cudaStreamWaitEvent(s, f->ev_join[j], 0));
    }
    for (int h = 1; h <= f->maxL; ++h) {
        HeightPlan& hp = f->H[h];
        FCK(merge_form_kform_batch(hp.d_forms, hp.nforms, hp.max_m, s));
        if (int rc = run_gemm(f, hp.M1, h, 1, tune, s)) return rc;     // B1 = -A2 T1_iN
        if (int rc = run_gemm(f, hp.K, h, 0, tune, s)) return rc;      // K -= A2 A1
        for (GJGroup& g : hp.gj) FCK(gj_invert_batch(g.d_desc, g.count, g.m, g.flags, f->d_status, s));
        if (int rc = run_gemm(f, hp.M2, h, 2, tune, s)) return rc;
        if (int rc = run_gemm(f, hp.M3, h, 3, tune, s)) return rc;
        if (int rc = run_gemm(f, hp.M4, h, 4, tune, s)) return rc;
    }
    return RB_OK;
}

}  // namespace

extern "C" {

int rb_forest_create(rb_tree* const* trees, int ntrees, rb_forest** out) {
    if (!trees || ntrees <= 0 || !out) {
        set_thread_error("rb_forest_create: needs at least one tree");
        return RB_ERR_INVALID;
    }
    *out = nullptr;
    rb_forest* f = new rb_forest();
    auto bail = [&](int rc, const std::string& msg) {
        set_thread_error(msg.c_str());
        rb_forest_destroy(f);
        return rc;
    };
    if (cudaGetDevice(&f->device) != cudaSuccess) return bail(RB_ERR_CUDA, "rb_forest_create: no CUDA device");
    for (int i = 0; i < ntrees; ++i) {
        rb_tree* t = trees[i];
        if (!t) return bail(RB_ERR_INVALID, "rb_forest_create: null tree");
        for (int j = 0; j < i; ++j)
            if (trees[j] == t) return bail(RB_ERR_INVALID, "rb_forest_create: a tree is listed twice");
        if (!t->kform)
            return bail(RB_ERR_UNSUPPORTED, "rb_forest_create: every tree needs the single-inversion (K form) merge");
        if (t->P.d != 2) return bail(RB_ERR_UNSUPPORTED, "rb_forest_create: forests of 3D trees are not implemented");
        if (int rc = tree_prepare_factor(t)) return bail(rc, "rb_forest_create: " + t->err);
        if (t->device != f->device) return bail(RB_ERR_INVALID, "rb_forest_create: trees on different devices");
        f->trees.push_back(t);
        f->maxL = std::max(f->maxL, t->P.L);
    }
    if (cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(RB_ERR_CUDA, "rb_forest_create: stream creation failed");
    const int nside = std::min(ntrees, 8);
    f->side.assign(nside, nullptr);
    f->ev_fork.assign(1, nullptr);
    f->ev_join.assign(nside, nullptr);
    bool ok = cudaEventCreateWithFlags(&f->ev_fork[0], cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreate(&f->ev0) == cudaSuccess && cudaEventCreate(&f->ev1) == cudaSuccess;
    for (int j = 0; ok && j < nside; ++j)
        ok = cudaStreamCreateWithFlags(&f->side[j], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&f->ev_join[j], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) return bail(RB_ERR_CUDA, "rb_forest_create: stream or event creation failed");
    void* p = nullptr;
    if (falloc(f, sizeof(int), &p)) return bail(RB_ERR_OUT_OF_MEMORY, f->err);
    f->d_status = static_cast<int*>(p);
    if (cudaMallocHost(&f->h_status, sizeof(int)) != cudaSuccess)
        return bail(RB_ERR_CUDA, "rb_forest_create: pinned allocation failed");
    if (int rc = build_plan(f)) return bail(rc, f->err);
    // a stage whose shape was tuned before (this process) takes the known choice
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        bool all = true;
        for (int h = 1; h <= f->maxL; ++h)
            for (GemmBatch* b : {&f->H[h].K, &f->H[h].M1, &f->H[h].M2, &f->H[h].M3, &f->H[h].M4}) {
                if (b->count == 0) continue;
                auto it = g_tuned.find(sig_of(*b));
                if (it != g_tuned.end()) b->engine = it->second;
                else all = false;
            }
        f->tuned = all;
    }
    *out = f;
    return RB_OK;
}

int rb_forest_destroy(rb_forest* f) {
    if (!f) return RB_OK;
    if (f->stream) cudaStreamSynchronize(f->stream);
    if (f->gx) cudaGraphExecDestroy(f->gx);
    for (void* p : f->bufs) cudaFree(p);
    for (auto e : f->ev_fork) if (e) cudaEventDestroy(e);
    for (auto e : f->ev_join) if (e) cudaEventDestroy(e);
    if (f->ev0) cudaEventDestroy(f->ev0);
    if (f->ev1) cudaEventDestroy(f->ev1);
    for (auto s : f->side) if (s) cudaStreamDestroy(s);
    if (f->stream) cudaStreamDestroy(f->stream);
    if (f->h_status) cudaFreeHost(f->h_status);
    delete f;
    return RB_OK;
}

const char* rb_forest_last_error(const rb_forest* f) { return f ? f->err.c_str() : rb_last_error(nullptr); }

int rb_forest_factor(rb_forest* f, const double* const* d_k, int autotune) {
    if (!f || !d_k) return RB_ERR_INVALID;
    cudaStream_t s = f->stream;
    // the potentials into each tree's own copy (the schedule reads t->d_k)
    for (size_t i = 0; i < f->trees.size(); ++i) {
        rb_tree* t = f->trees[i];
        if (!d_k[i]) {
            f->err = "rb_forest_factor: null potential";
            return RB_ERR_INVALID;
        }
        const size_t nint = (size_t)t->P.nleaves() * t->P.leaf_a() * t->P.leaf_b();
        FCK(cudaMemcpyAsync(t->d_k, d_k[i], nint * sizeof(z), cudaMemcpyDeviceToDevice, s));
    }
    if (autotune && !f->tuned) {
        if (int rc = run_schedule(f, true)) return rc;       // tuning pass: results discarded
        FCK(cudaStreamSynchronize(s));
        f->tuned = true;
        if (f->gx) {
            cudaGraphExecDestroy(f->gx);
            f->gx = nullptr;
        }
        f->runs = 0;
    }
    const long long l0 = launch_count();
    FCK(cudaEventRecord(f->ev0, s));
    if (f->runs == 0) {
        if (int rc = run_schedule(f, false)) return rc;
        f->launches = launch_count() - l0;
    } else {
        if (!f->gx) {
            FCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            const long long c0 = launch_count();
            const int rc = run_schedule(f, false);
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(s, &g);
            if (rc || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                if (rc) return rc;
                f->err = std::string("forest graph capture failed: ") + cudaGetErrorString(e);
                return RB_ERR_CUDA;
            }
            f->launches = launch_count() - c0;
            const cudaError_t ei = cudaGraphInstantiate(&f->gx, g, 0);
            cudaGraphDestroy(g);
            if (ei != cudaSuccess) {
                f->gx = nullptr;
                f->err = std::string("forest graph instantiation failed: ") + cudaGetErrorString(ei);
                return RB_ERR_CUDA;
            }
        }
        FCK(cudaGraphLaunch(f->gx, s));
    }
    ++f->runs;
    FCK(cudaMemcpyAsync(f->h_status, f->d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
    FCK(cudaEventRecord(f->ev1, s));
    FCK(cudaEventSynchronize(f->ev1));
    float ms = 0.f;
    FCK(cudaEventElapsedTime(&ms, f->ev0, f->ev1));
    f->f_time = ms * 1e-3;
    if (*f->h_status) {
        f->err = (*f->h_status & (RB_STATUS_GJ_TIMEOUT | RB_TC5_TIMEOUT)) ? "a device wait timed out in the forest factor"
                                                                          : "zero pivot met in the forest factor";
        return (*f->h_status & RB_STATUS_ZERO_PIVOT) ? RB_ERR_NUMERIC : RB_ERR_CUDA;
    }
    for (rb_tree* t : f->trees) tree_mark_factored(t, f->f_time);
    return RB_OK;
}

int rb_forest_info(const rb_forest* f, double* f_time, int64_t* launches, int32_t* tuned_stages) {
    if (!f) return RB_ERR_INVALID;
    if (f_time) *f_time = f->f_time;
    if (launches) *launches = f->launches;
    if (tuned_stages) {
        int n = 0;
        for (int h = 1; h <= f->maxL; ++h)
            for (const GemmBatch* b : {&f->H[h].K, &f->H[h].M1, &f->H[h].M2, &f->H[h].M3, &f->H[h].M4})
                if (b->count && b->engine >= 0) ++n;
        *tuned_stages = n;
    }
    return RB_OK;
}

int rb_forest_tuning(const rb_forest* f, int32_t* height, int32_t* stage, int32_t* engine, double* ms, int n) {
    if (!f) return RB_ERR_INVALID;
    const int cnt = (int)f->tune_log.size();
    for (int i = 0; i < std::min(n, cnt); ++i) {
        if (height) height[i] = f->tune_log[i].h;
        if (stage) stage[i] = f->tune_log[i].stage;
        if (engine) engine[i] = f->tune_log[i].engine;
        if (ms) ms[i] = f->tune_log[i].ms;
    }
    return cnt;
}

const char* rb_gemm_engine_name(int engine) { return gemm_engine_name(engine); }

}  // extern "C"
