// rb_server.cpp -- serving loop over resident factorized trees (include/robin_b200.h, rb_server_*).
//
// The reference factors one tree and solves one right-hand side per call, once per process
// (robin_tree_solve, robin_tree_module.f90:198-233; boundary data only on the first solve,
// :1014-1029).  This server keeps several factorized trees resident in device memory and serves a
// stream of factor and solve requests against them:
//   * one worker thread per tree owns the tree's handle (its CUDA streams); trees run their work
//     concurrently on the device;
//   * continuous batching: the solve requests queued for a tree when its worker becomes free are
//     merged, up to max_batch_rhs right-hand sides, into ONE batched up/down sweep; requests that
//     arrive meanwhile form the next batch.  A batch is padded with zero right-hand sides to a
//     power of two, so that each tree reuses a few cached launch plans (one per RHS count).  A factor request is a barrier in its tree's queue:
//     solves submitted before it use the old factorization, solves after it the new one;
//   * admission by device memory: a tree's first factorization reserves its estimated footprint
//     (factor storage, solve buffers of a full batch, input staging) against the server's budget
//     and waits while the other trees' reservations leave too little room;
//   * inputs are either host arrays or standard fields sampled on the device
//     (rb_tree_sample_device: point sources, plane waves, bump potentials), so a request's
//     sources need not cross PCIe; solutions are copied to the caller's host buffer;
//   * latency = arrival (the caller's stamp on the server clock, or the submit time) to the
//     request's completion with its solution in host memory.
// Batched right-hand sides of an FP64 tree are bit-identical to the same right-hand sides solved
// alone (the solve's GEMMs sum in an order independent of the batch); a mixed-precision tree
// refines each batch to the server's tolerance.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "robin_b200.h"
#include "rb_kernels.h"

namespace rb {
const z* tree_solutions(const rb_tree* t);
double tree_bytes_estimate(const rb_tree* t, int nrhs, int precision);
}  // namespace rb

using namespace rb;

namespace {

using Clock = std::chrono::steady_clock;

enum { REQ_FACTOR = 0, REQ_SOLVE = 1 };

struct Request {
    int64_t id = 0;
    int kind = REQ_SOLVE;
    int tree = 0;
    int nrhs = 0;
    int field = -1;                 // RB_FIELD_* sampled on the device, or -1: host arrays
    std::vector<double> params;     // field parameters (copied at submit)
    std::vector<double> k;          // factor: host potential samples (copied at submit)
    const double* f = nullptr;      // solve, host inputs: read until completion (NULL = zero)
    const double* g = nullptr;
    double* u = nullptr;            // solve: host output (NULL: not copied)
    double arrival = 0.0, done = 0.0;
    int status = RB_OK;
    std::string err;
    bool finished = false;
};
using ReqPtr = std::shared_ptr<Request>;

struct TreeSlot {
    int id = 0;
    rb_tree* t = nullptr;
    rb_info info{};
    std::deque<ReqPtr> queue;
    std::condition_variable cv;
    std::thread worker;
    bool factored = false;
    double reserved = 0.0;          // bytes reserved against the server budget
    double* f_stage = nullptr;      // max_batch_rhs * n_interior complex
    double* g_stage = nullptr;      // max_batch_rhs * root_nb complex
    double* k_stage = nullptr;      // n_interior complex
};

}  // namespace

struct rb_server {
    rb_server_opts opts{};
    int device = 0;
    double budget = 0.0;
    double reserved_total = 0.0;
    std::mutex mu;
    std::condition_variable done_cv;
    std::condition_variable mem_cv;
    std::vector<std::unique_ptr<TreeSlot>> trees;
    std::unordered_map<int64_t, ReqPtr> reqs;
    int64_t next_id = 1;
    bool stop = false;
    Clock::time_point t0;
    std::string err;
    // statistics since the last reset
    std::vector<double> solve_lat, factor_lat;
    int64_t n_solves = 0, n_rhs = 0, n_factors = 0, n_batches = 0, n_failed = 0;
};

static double now_s(const rb_server* s) {
    return std::chrono::duration<double>(Clock::now() - s->t0).count();
}

static void finish(rb_server* s, const ReqPtr& r, int status, const std::string& msg) {
    // called with s->mu held
    r->status = status;
    r->err = msg;
    r->done = now_s(s);
    r->finished = true;
    if (status != RB_OK) {
        ++s->n_failed;
    } else if (r->kind == REQ_SOLVE) {
        ++s->n_solves;
        s->n_rhs += r->nrhs;
        s->solve_lat.push_back(r->done - r->arrival);
    } else {
        ++s->n_factors;
        s->factor_lat.push_back(r->done - r->arrival);
    }
    s->done_cv.notify_all();
}

static std::string cuda_msg(const char* what, cudaError_t e) { return std::string(what) + ": " + cudaGetErrorString(e); }

// Reserves the tree's footprint against the budget (waits while other trees hold too much) and
// allocates its staging buffers.  Called with the lock held; returns with it held.
static int admit(rb_server* s, TreeSlot& slot, std::unique_lock<std::mutex>& lk, std::string& msg) {
    if (slot.reserved > 0.0) return RB_OK;
    const int B = s->opts.max_batch_rhs;
    const double stage = ((double)B * slot.info.n_interior + (double)B * slot.info.root_nb + slot.info.n_interior) * 16.0;
    const double need = tree_bytes_estimate(slot.t, B, s->opts.precision) + stage;
    if (need > s->budget) {
        msg = "tree needs about " + std::to_string((long long)need) + " bytes of device memory, the server's budget is " +
              std::to_string((long long)s->budget);
        return RB_ERR_OUT_OF_MEMORY;
    }
    s->mem_cv.wait(lk, [&] { return s->stop || s->reserved_total + need <= s->budget; });
    if (s->stop) {
        msg = "server stopped";
        return RB_ERR_INVALID;
    }
    s->reserved_total += need;
    slot.reserved = need;
    lk.unlock();
    cudaError_t e = cudaMalloc(&slot.f_stage, (size_t)B * slot.info.n_interior * 16);
    if (e == cudaSuccess) e = cudaMalloc(&slot.g_stage, (size_t)B * slot.info.root_nb * 16);
    if (e == cudaSuccess) e = cudaMalloc(&slot.k_stage, (size_t)slot.info.n_interior * 16);
    lk.lock();
    if (e != cudaSuccess) {
        cudaGetLastError();
        msg = cuda_msg("staging allocation failed", e);
        return RB_ERR_OUT_OF_MEMORY;
    }
    return RB_OK;
}

static void run_factor_request(rb_server* s, TreeSlot& slot, const ReqPtr& r, std::unique_lock<std::mutex>& lk) {
    std::string msg;
    int rc = admit(s, slot, lk, msg);
    if (rc) {
        finish(s, r, rc, msg);
        return;
    }
    lk.unlock();
    if (r->field >= 0) {
        rc = rb_tree_sample_device(slot.t, RB_FIELD_BUMP_POTENTIAL, (int)(r->params.size() - 3) / 3, r->params.data(),
                                   slot.k_stage, nullptr, 0);
        if (!rc) rc = rb_tree_factor_device(slot.t, slot.k_stage, s->opts.precision, 1);
    } else {
        rc = rb_tree_factor(slot.t, r->k.data(), s->opts.precision);
    }
    if (!rc && s->opts.precision == RB_PREC_MIXED) rc = rb_tree_set_refinement(slot.t, s->opts.tol, 8);
    msg = rc ? rb_last_error(slot.t) : "";
    lk.lock();
    slot.factored = rc == RB_OK;
    finish(s, r, rc, msg);
}

static void run_solve_batch(rb_server* s, TreeSlot& slot, std::vector<ReqPtr>& batch, std::unique_lock<std::mutex>& lk) {
    if (!slot.factored) {
        for (auto& r : batch) finish(s, r, RB_ERR_NOT_FACTORED, "Error: Robin Tree must be factored first.");
        return;
    }
    lk.unlock();
    const int64_t nint = slot.info.n_interior, nb = slot.info.root_nb;
    const size_t per = (size_t)slot.info.nleaves * slot.info.leaf_n;
    cudaStream_t st = static_cast<cudaStream_t>(rb_tree_stream(slot.t));
    int rc = RB_OK;
    std::string msg;
    int tot = 0;
    for (auto& r : batch) {
        double* fo = slot.f_stage + 2 * (size_t)tot * nint;
        double* go = slot.g_stage + 2 * (size_t)tot * nb;
        if (r->field >= 0) {
            rc = rb_tree_sample_device(slot.t, r->field, r->nrhs, r->params.data(), fo, go, 0);
            if (rc) msg = rb_last_error(slot.t);
        } else {
            cudaError_t e = r->f ? cudaMemcpyAsync(fo, r->f, (size_t)r->nrhs * nint * 16, cudaMemcpyHostToDevice, st)
                                 : cudaMemsetAsync(fo, 0, (size_t)r->nrhs * nint * 16, st);
            if (e == cudaSuccess)
                e = r->g ? cudaMemcpyAsync(go, r->g, (size_t)r->nrhs * nb * 16, cudaMemcpyHostToDevice, st)
                         : cudaMemsetAsync(go, 0, (size_t)r->nrhs * nb * 16, st);
            if (e != cudaSuccess) {
                rc = RB_ERR_CUDA;
                msg = cuda_msg("input copy failed", e);
            }
        }
        if (rc) break;
        tot += r->nrhs;
    }
    // the batch is padded with zero right-hand sides up to a power of two (at most max_batch_rhs):
    // a tree then solves at most a handful of distinct RHS counts, whose launch plans and graphs
    // it keeps, instead of building one for nearly every batch.  Every right-hand side is solved
    // independently, so the padding changes no result.
    int padded = tot;
    if (!rc && tot > 0) {
        padded = 1;
        while (padded < tot) padded *= 2;
        padded = std::min(padded, std::max(tot, s->opts.max_batch_rhs));
        if (padded > tot) {
            cudaError_t e = cudaMemsetAsync(slot.f_stage + 2 * (size_t)tot * nint, 0, (size_t)(padded - tot) * nint * 16, st);
            if (e == cudaSuccess)
                e = cudaMemsetAsync(slot.g_stage + 2 * (size_t)tot * nb, 0, (size_t)(padded - tot) * nb * 16, st);
            if (e != cudaSuccess) {
                rc = RB_ERR_CUDA;
                msg = cuda_msg("batch padding failed", e);
            }
        }
    }
    if (!rc) {
        rc = rb_tree_solve_device(slot.t, padded, slot.f_stage, slot.g_stage, 0);
        if (rc) msg = rb_last_error(slot.t);
    }
    if (!rc) {
        const z* sol = tree_solutions(slot.t);
        int o = 0;
        for (auto& r : batch) {
            if (r->u) {
                cudaError_t e = cudaMemcpyAsync(r->u, sol + (size_t)o * per, (size_t)r->nrhs * per * 16,
                                                cudaMemcpyDeviceToHost, st);
                if (e != cudaSuccess) {
                    rc = RB_ERR_CUDA;
                    msg = cuda_msg("solution copy failed", e);
                    break;
                }
            }
            o += r->nrhs;
        }
        cudaError_t e = cudaStreamSynchronize(st);
        if (!rc && e != cudaSuccess) {
            rc = RB_ERR_CUDA;
            msg = cuda_msg("solve failed", e);
        }
    }
    lk.lock();
    ++s->n_batches;
    for (auto& r : batch) finish(s, r, rc, msg);
}

static void worker_main(rb_server* s, TreeSlot* slot) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        slot->cv.wait(lk, [&] { return s->stop || !slot->queue.empty(); });
        if (s->stop) break;
        ReqPtr front = slot->queue.front();
        if (front->kind == REQ_FACTOR) {
            slot->queue.pop_front();
            run_factor_request(s, *slot, front, lk);
            continue;
        }
        std::vector<ReqPtr> batch;
        int tot = 0;
        while (!slot->queue.empty() && slot->queue.front()->kind == REQ_SOLVE) {
            const ReqPtr& r = slot->queue.front();
            if (tot > 0 && tot + r->nrhs > s->opts.max_batch_rhs) break;
            tot += r->nrhs;
            batch.push_back(r);
            slot->queue.pop_front();
        }
        run_solve_batch(s, *slot, batch, lk);
    }
    // drain: requests still queued are refused
    for (auto& r : slot->queue) finish(s, r, RB_ERR_INVALID, "server stopped");
    slot->queue.clear();
}

static int srv_fail(rb_server* s, int code, const std::string& msg) {
    std::lock_guard<std::mutex> g(s->mu);
    s->err = msg;
    return code;
}

extern "C" {

int rb_server_create(const rb_server_opts* opts, rb_server** out) {
    if (!out) return RB_ERR_INVALID;
    *out = nullptr;
    rb_server_opts o{};
    if (opts) o = *opts;
    if (o.max_batch_rhs <= 0) o.max_batch_rhs = 64;
    if (o.tol <= 0.0) o.tol = 1e-10;
    if (o.precision != RB_PREC_FP64 && o.precision != RB_PREC_MIXED) {
        set_thread_error("rb_server_create: precision must be RB_PREC_FP64 or RB_PREC_MIXED");
        return RB_ERR_INVALID;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        set_thread_error("rb_server_create: no CUDA device");
        return RB_ERR_CUDA;
    }
    double budget = (double)o.device_budget;
    if (budget <= 0.0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            set_thread_error("rb_server_create: cudaMemGetInfo failed");
            return RB_ERR_CUDA;
        }
        budget = 0.9 * (double)fr;
    }
    rb_server* s = new rb_server();
    s->opts = o;
    s->device = dev;
    s->budget = budget;
    s->t0 = Clock::now();
    *out = s;
    return RB_OK;
}

int rb_server_destroy(rb_server* s) {
    if (!s) return RB_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        for (auto& t : s->trees) t->cv.notify_all();
        s->mem_cv.notify_all();
    }
    for (auto& t : s->trees)
        if (t->worker.joinable()) t->worker.join();
    for (auto& t : s->trees) {
        if (t->t) rb_tree_destroy(t->t);
        cudaFree(t->f_stage);
        cudaFree(t->g_stage);
        cudaFree(t->k_stage);
    }
    delete s;
    return RB_OK;
}

const char* rb_server_last_error(const rb_server* s) { return s ? s->err.c_str() : rb_last_error(nullptr); }

double rb_server_now(const rb_server* s) { return s ? now_s(s) : 0.0; }

int rb_server_add_tree(rb_server* s, const rb_geom* geom, int32_t* tree_id) {
    if (!s || !geom || !tree_id) return RB_ERR_INVALID;
    rb_geom g = *geom;
    g.device_budget = 0;                       // the server's budget governs
    g.flags &= ~RB_FLAG_ASYNC_FACTOR;
    rb_tree* t = nullptr;
    int rc = rb_tree_create(&g, &t);
    if (rc) return srv_fail(s, rc, rb_last_error(nullptr));
    auto slot = std::make_unique<TreeSlot>();
    slot->t = t;
    rb_tree_info(t, &slot->info);
    std::lock_guard<std::mutex> lk(s->mu);
    slot->id = (int)s->trees.size();
    *tree_id = slot->id;
    TreeSlot* raw = slot.get();
    s->trees.push_back(std::move(slot));
    raw->worker = std::thread(worker_main, s, raw);
    return RB_OK;
}

int rb_server_tree_info(rb_server* s, int32_t tree_id, rb_info* info) {
    if (!s || !info) return RB_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    if (tree_id < 0 || tree_id >= (int)s->trees.size()) return RB_ERR_INVALID;
    *info = s->trees[tree_id]->info;
    return RB_OK;
}

static int submit(rb_server* s, ReqPtr r, int64_t* req) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (r->tree < 0 || r->tree >= (int)s->trees.size()) {
        s->err = "unknown tree id " + std::to_string(r->tree);
        return RB_ERR_INVALID;
    }
    if (s->stop) {
        s->err = "server stopped";
        return RB_ERR_INVALID;
    }
    r->id = s->next_id++;
    if (r->arrival < 0.0) r->arrival = now_s(s);
    s->reqs[r->id] = r;
    TreeSlot& slot = *s->trees[r->tree];
    slot.queue.push_back(r);
    slot.cv.notify_one();
    *req = r->id;
    return RB_OK;
}

int rb_server_submit_factor(rb_server* s, int32_t tree, const double* k, int field_count, const double* field_params,
                            double arrival, int64_t* req) {
    if (!s || !req) return RB_ERR_INVALID;
    auto r = std::make_shared<Request>();
    r->kind = REQ_FACTOR;
    r->tree = tree;
    r->arrival = arrival;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (tree < 0 || tree >= (int)s->trees.size()) {
            s->err = "unknown tree id " + std::to_string(tree);
            return RB_ERR_INVALID;
        }
        if (k) {
            r->k.assign(k, k + 2 * s->trees[tree]->info.n_interior);
        } else {
            if (field_count < 0 || !field_params) {
                s->err = "rb_server_submit_factor: needs host samples or bump-potential parameters";
                return RB_ERR_INVALID;
            }
            r->field = RB_FIELD_BUMP_POTENTIAL;
            r->params.assign(field_params, field_params + 3 + 3 * (size_t)field_count);
        }
    }
    return submit(s, r, req);
}

int rb_server_submit_solve(rb_server* s, int32_t tree, int nrhs, int field, const double* params, const double* f,
                           const double* g, double* u, double arrival, int64_t* req) {
    if (!s || !req) return RB_ERR_INVALID;
    if (nrhs <= 0 || nrhs > s->opts.max_batch_rhs)
        return srv_fail(s, RB_ERR_INVALID, "rb_server_submit_solve: nrhs must be in 1..max_batch_rhs");
    auto r = std::make_shared<Request>();
    r->kind = REQ_SOLVE;
    r->tree = tree;
    r->nrhs = nrhs;
    r->arrival = arrival;
    r->u = u;
    if (field >= 0) {
        if ((field != RB_FIELD_POINT_SOURCE && field != RB_FIELD_PLANE_WAVE) || !params)
            return srv_fail(s, RB_ERR_INVALID, "rb_server_submit_solve: field must be a point source or plane wave");
        r->field = field;
        r->params.assign(params, params + 3 * (size_t)nrhs);
    } else {
        r->f = f;
        r->g = g;
    }
    return submit(s, r, req);
}

int rb_server_wait(rb_server* s, int64_t req, double timeout_s) {
    if (!s) return RB_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(req);
    if (it == s->reqs.end()) {
        s->err = "unknown or already collected request " + std::to_string(req);
        return RB_ERR_INVALID;
    }
    ReqPtr r = it->second;
    auto pred = [&] { return r->finished; };
    if (timeout_s < 0.0) s->done_cv.wait(lk, pred);
    else if (!s->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) return 1;
    s->reqs.erase(req);
    if (r->status) s->err = r->err;
    return r->status;
}

int rb_server_get_stats(rb_server* s, rb_server_stats* out, int reset) {
    if (!s || !out) return RB_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->solves = s->n_solves;
    out->rhs = s->n_rhs;
    out->factors = s->n_factors;
    out->batches = s->n_batches;
    out->failed = s->n_failed;
    auto pct = [](std::vector<double> v, double q) {
        if (v.empty()) return 0.0;
        std::sort(v.begin(), v.end());
        const size_t i = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
        return v[i] * 1e3;
    };
    out->p50_ms = pct(s->solve_lat, 0.50);
    out->p99_ms = pct(s->solve_lat, 0.99);
    out->max_ms = pct(s->solve_lat, 1.0);
    double sum = 0.0;
    for (double v : s->solve_lat) sum += v;
    out->mean_ms = s->solve_lat.empty() ? 0.0 : 1e3 * sum / (double)s->solve_lat.size();
    out->factor_p50_ms = pct(s->factor_lat, 0.50);
    out->factor_max_ms = pct(s->factor_lat, 1.0);
    out->reserved_bytes = (int64_t)s->reserved_total;
    if (reset) {
        s->solve_lat.clear();
        s->factor_lat.clear();
        s->n_solves = s->n_rhs = s->n_factors = s->n_batches = s->n_failed = 0;
    }
    return RB_OK;
}

}  // extern "C"
