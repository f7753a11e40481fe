// Solve service on one GPU: continuous batching of uneven requests on top of
// the batched engine (batch.cu). No counterpart in the reference, which runs
// one scenario per process (src/Main.cpp:1193-1227).
//
// One scheduler thread owns the batch. Its loop:
//   1. if a run is in flight and has ended: harvest finished instances and
//      complete their requests;
//   2. add the instances set up meanwhile, and relaunch the graph (it stops
//      by itself when an instance finishes or after trip_quantum trips);
//   3. while the graph runs: admit pending requests in arrival order while
//      their footprint fits the free device memory minus the reserve, build
//      each one's instance on the set-up stream (overlapping the graph), and
//      once some are ready make the graph stop at its next trip boundary so
//      that they join.
// Submitters and waiters only touch the queues under the mutex.
//
// FP64 (and floatBoost) requests take the same admission path but are solved
// by cp_solve, one request per lane thread; each lane has its own context
// (stream), so the lanes' solves and the batch run concurrently. A small
// request's CG occupies one 16-SM cluster, so several of them share the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "instance.h"
#include "internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    long long id = 0;
    int nn = 0, c3 = 0, c4 = 0, c8 = 0;
    std::vector<double> xy, rp, uv;
    std::vector<int> e3, e4, e8;
    std::vector<unsigned char> mask;
    bool has_uv = false;
    cp_material mat{};
    cp_solve_opts opts{};
    size_t footprint = 0;
    Clock::time_point t_submit, t_done;
    cp_instance* inst = nullptr;
    cp_solve_report rep{};
    int status = CP_OK;  // set-up or cancellation error
    bool done = false;
};

using ReqP = std::shared_ptr<Request>;

}  // namespace

struct cp_server {
    cp_server_opts o{};
    cp_context* ctx_run = nullptr;
    cp_context* ctx_setup = nullptr;
    cp_batch* batch = nullptr;
    std::vector<cp_context*> lane_ctx;    // one per FP64 lane
    // Oldest first: each lane has one stream per priority level, and the
    // running requests in submission order take the levels from the highest
    // down (the last level shared by the rest), reassigned whenever a lane
    // starts or ends a request; a running solve moves to its new stream at
    // its next outer iteration. lane_own[k] is the stream lane_ctx[k] was
    // created with (restored before the context is destroyed).
    std::vector<std::vector<cudaStream_t>> lane_streams;
    std::vector<cudaStream_t> lane_own;
    std::vector<int> lane_level;          // the level each lane's request runs at (-1: idle)
    // The context of every instance handed back to a caller: the lanes' and
    // the set-up contexts keep working (and capture CUDA graphs on their
    // streams) while callers read results, so a result moves to this
    // context, whose stream only the callers use, before it is handed over.
    cp_context* ctx_out = nullptr;
    std::vector<std::thread> lanes;
    std::deque<ReqP> lane_q;              // admitted FP64 requests, not yet on a lane
    std::vector<ReqP> lane_cur;           // the request each lane is solving (or null)
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_lane;
    std::deque<ReqP> pending;
    std::unordered_map<long long, ReqP> by_id;         // submitted, not yet taken
    std::unordered_map<cp_instance*, ReqP> inflight;   // in the batch or set up, waiting to join
    long long next_id = 1;
    bool stop = false;
    std::thread th;
    cp_server_stats st{};
    size_t inflight_bytes = 0;
    size_t total_mem = 0;
};

namespace {

// Live servers. At process exit their scheduler threads are stopped and
// joined before the CUDA runtime tears down (the handler is registered after
// the runtime initialised, so it runs first); nothing is freed there.
std::mutex g_live_mu;
std::vector<cp_server*> g_live;
bool g_atexit_registered = false;

void stop_thread(cp_server* s) {
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        for (auto& r : s->lane_cur)  // the lanes' solves stop at their next outer iteration
            if (r && r->inst) r->inst->cancel.store(1);
    }
    cp_batch_interrupt(s->batch);
    s->cv_work.notify_all();
    s->cv_lane.notify_all();
    if (s->th.joinable()) s->th.join();
    for (auto& t : s->lanes)
        if (t.joinable()) t.join();
}

bool is_lane_request(const cp_solve_opts& o) { return o.precision != CP_PREC_MIXED; }

// Reassigns the levels of the running requests (s->mu held).
void relevel(cp_server* s) {
    if (s->lane_streams.empty()) return;
    std::vector<std::pair<long long, int>> run;
    for (size_t j = 0; j < s->lane_cur.size(); ++j)
        if (s->lane_cur[j]) run.emplace_back(s->lane_cur[j]->id, (int)j);
        else s->lane_level[j] = -1;
    std::sort(run.begin(), run.end());
    for (size_t i = 0; i < run.size(); ++i) {
        const int j = run[i].second;
        const int lv = (int)std::min(i, s->lane_streams[j].size() - 1);
        if (lv != s->lane_level[j]) {
            s->lane_level[j] = lv;
            s->lane_ctx[j]->restream.store(s->lane_streams[j][lv]);
        }
    }
}

// Gives every lane context its own stream back and destroys the priority
// streams (before the lane contexts are destroyed).
void release_lane_streams(cp_server* s) {
    for (size_t k = 0; k < s->lane_own.size() && k < s->lane_ctx.size(); ++k) {
        cudaStreamSynchronize(s->lane_ctx[k]->stream);
        s->lane_ctx[k]->stream = s->lane_own[k];
    }
    for (auto& v : s->lane_streams)
        for (cudaStream_t st : v) cudaStreamDestroy(st);
    for (cp_context* c : s->lane_ctx) c->restream.store(nullptr);
    s->lane_streams.clear();
    s->lane_own.clear();
}

void stop_all_at_exit() {
    std::lock_guard<std::mutex> lock(g_live_mu);
    for (cp_server* s : g_live) stop_thread(s);
}

void complete(cp_server* s, const ReqP& r) {
    r->t_done = Clock::now();
    r->done = true;
    if (r->status != CP_OK || r->rep.status != CP_OK) s->st.failed += 1;
    s->st.completed += 1;
}

// Builds the instance of a request on stream ctx (the set-up stream for the
// batch, the lane's own for an FP64 request) into *out; the caller publishes
// it in the request under the mutex.
int setup(cp_context* ctx, const ReqP& r, cp_instance** out) {
    *out = nullptr;
    cp_mesh_view v{};
    v.node_count = r->nn;
    v.node_xy = r->xy.data();
    v.count3 = r->c3;
    v.elem3 = r->c3 ? r->e3.data() : nullptr;
    v.count4 = r->c4;
    v.elem4 = r->c4 ? r->e4.data() : nullptr;
    v.count8 = r->c8;
    v.elem8 = r->c8 ? r->e8.data() : nullptr;
    cp_instance* I = nullptr;
    int st = cp_instance_create(ctx, &v, &r->mat, &I);
    if (st != CP_OK) return st;
    st = cp_instance_set_loads(I, r->rp.data(), r->mask.data(), r->has_uv ? r->uv.data() : nullptr);
    if (st == CP_OK && !is_lane_request(r->opts)) {
        try {
            cp::instance_prepare_mixed(I, r->opts.precond);
            if (cudaStreamSynchronize(I->s()) != cudaSuccess) st = CP_ERR_CUDA;
        } catch (const cp::Error& e) {
            st = e.status;
        }
    }
    if (st != CP_OK) {
        cp_instance_destroy(I);
        return st;
    }
    *out = I;
    return CP_OK;
}

// One FP64 lane: takes admitted requests in order and solves each with
// cp_solve on its own stream.
void lane(cp_server* s, int k) {
    cudaSetDevice(s->o.device);
    for (;;) {
        ReqP r;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            s->cv_lane.wait(lock, [&] { return s->stop || !s->lane_q.empty(); });
            if (s->stop) return;
            r = s->lane_q.front();
            s->lane_q.pop_front();
            s->lane_cur[k] = r;
            if (!s->lane_streams.empty()) {
                s->lane_level[k] = -1;
                relevel(s);
                // this lane's stream is idle between requests: take the level now
                s->lane_ctx[k]->restream.store(nullptr);
                s->lane_ctx[k]->stream = s->lane_streams[k][s->lane_level[k]];
            }
        }
        cp_instance* inst = nullptr;
        int rc = setup(s->lane_ctx[k], r, &inst);
        cp_solve_report rep{};
        if (rc == CP_OK) {
            {
                std::lock_guard<std::mutex> lock(s->mu);
                r->inst = inst;
                if (s->stop) inst->cancel.store(1);
            }
            const int st = cp_solve(inst, &r->opts, &rep);
            if (st != CP_OK && rep.status == CP_OK) rep.status = st;
            // nothing of this instance stays in flight on the lane's stream
            if (cudaStreamSynchronize(inst->ctx->stream) != cudaSuccess && rep.status == CP_OK) rep.status = CP_ERR_CUDA;
            inst->ctx = s->ctx_out;
        }
        std::lock_guard<std::mutex> lock(s->mu);
        s->lane_cur[k] = nullptr;
        relevel(s);
        s->inflight_bytes -= r->footprint;
        if (rc != CP_OK) {
            r->status = rc;
        } else {
            r->rep = rep;
            if (rep.status == CP_ERR_CANCELLED) r->status = CP_ERR_CANCELLED;
        }
        complete(s, r);
        s->cv_done.notify_all();
        s->cv_work.notify_all();  // memory and a slot are free again
    }
}

void scheduler(cp_server* s) {
    cudaSetDevice(s->o.device);
    bool running = false;
    std::vector<ReqP> ready;  // set up, waiting to join the batch
    Clock::time_point t_launch;
    const size_t reserve = (size_t)(s->o.hbm_reserve * (double)s->total_mem);
    for (;;) {
        if (running) {
            int active = 0, done = 0;
            const int rc = cp_batch_wait(s->batch, &active, &done);
            running = false;
            std::lock_guard<std::mutex> lock(s->mu);
            s->st.busy_seconds += std::chrono::duration<double>(Clock::now() - t_launch).count();
            cp_batch_stats(s->batch, &s->st.trips, nullptr, nullptr);
            std::vector<int> slots(s->inflight.size() + 1);
            std::vector<cp_instance*> insts(slots.size());
            std::vector<cp_solve_report> reps(slots.size());
            int n = 0;
            if (rc == CP_OK) cp_batch_harvest(s->batch, (int)slots.size(), slots.data(), insts.data(), reps.data(), &n);
            for (int i = 0; i < n; ++i) {
                auto it = s->inflight.find(insts[i]);
                if (it == s->inflight.end()) continue;
                ReqP r = it->second;
                s->inflight.erase(it);
                s->inflight_bytes -= r->footprint;
                r->rep = reps[i];
                if (r->inst) {  // the run has ended: hand the instance over on the callers' context
                    cudaStreamSynchronize(r->inst->ctx->stream);
                    r->inst->ctx = s->ctx_out;
                }
                complete(s, r);
            }
            if (rc != CP_OK) {
                // the device failed: fail everything still on it
                for (auto& kv : s->inflight) {
                    kv.second->status = rc;
                    complete(s, kv.second);
                }
                s->inflight.clear();
                s->inflight_bytes = 0;
                s->stop = true;
            }
            if (n > 0 || rc != CP_OK) s->cv_done.notify_all();
        }
        {
            std::lock_guard<std::mutex> lock(s->mu);
            if (s->stop) break;
        }
        // join the instances set up meanwhile and relaunch
        for (auto& r : ready) {
            int slot = -1;
            const int rc = cp_batch_add(s->batch, r->inst, &r->opts, &slot);
            if (rc != CP_OK) {
                std::lock_guard<std::mutex> lock(s->mu);
                s->inflight.erase(r->inst);
                s->inflight_bytes -= r->footprint;
                cp_instance_destroy(r->inst);
                r->inst = nullptr;
                r->status = rc;
                complete(s, r);
                s->cv_done.notify_all();
            }
        }
        ready.clear();
        int active = 0, done = 0;
        cp_batch_wait(s->batch, &active, &done);  // not running: counts only
        if (active > 0) {
            if (cp_batch_launch(s->batch, CP_BATCH_RUN_ANY_DONE, s->o.trip_quantum) == CP_OK) {
                running = true;
                t_launch = Clock::now();
                std::lock_guard<std::mutex> lock(s->mu);
                s->st.runs += 1;
            }
        }
        // admission while the graph runs (or while idle, block for work)
        for (;;) {
            std::vector<ReqP> take;
            {
                std::unique_lock<std::mutex> lock(s->mu);
                if (!running && ready.empty()) {
                    if (s->pending.empty())
                        s->cv_work.wait(lock, [&] { return s->stop || !s->pending.empty(); });
                    else  // waiting for memory that a caller still holds
                        s->cv_work.wait_for(lock, std::chrono::milliseconds(1));
                }
                if (s->stop) break;
                size_t free_b = 0, total_b = 0;
                cudaMemGetInfo(&free_b, &total_b);
                size_t planned = 0;
                int lane_busy = 0;
                for (auto& r : s->lane_cur) lane_busy += r ? 1 : 0;
                while (!s->pending.empty() && (int)(s->inflight.size() + s->lane_q.size() + lane_busy + take.size()) <
                                                  s->o.max_inflight) {
                    const ReqP& r = s->pending.front();
                    if (free_b < reserve || r->footprint + planned > free_b - reserve) break;  // head of line waits
                    if (s->o.max_bytes && s->inflight_bytes + planned + r->footprint > s->o.max_bytes) break;
                    planned += r->footprint;
                    take.push_back(r);
                    s->pending.pop_front();
                }
                for (auto& r : take) {
                    s->inflight_bytes += r->footprint;
                    s->st.admitted += 1;
                }
                if (s->inflight_bytes > s->st.peak_bytes) s->st.peak_bytes = s->inflight_bytes;
            }
            for (auto& r : take) {
                if (is_lane_request(r->opts)) {
                    std::lock_guard<std::mutex> lock(s->mu);
                    s->lane_q.push_back(r);
                    s->cv_lane.notify_one();
                    continue;
                }
                cp_instance* inst = nullptr;
                const int rc = setup(s->ctx_setup, r, &inst);
                std::lock_guard<std::mutex> lock(s->mu);
                r->inst = inst;
                if (rc == CP_OK) {
                    s->inflight[r->inst] = r;
                    ready.push_back(r);
                } else {
                    s->inflight_bytes -= r->footprint;
                    r->status = rc;
                    complete(s, r);
                    s->cv_done.notify_all();
                }
            }
            if (!running) break;  // nothing on the device: go and launch the ready ones
            if (!ready.empty()) {
                cp_batch_interrupt(s->batch);  // let them join at the next trip boundary
                break;
            }
            if (cudaStreamQuery(s->ctx_run->stream) != cudaErrorNotReady) break;  // the run ended
            std::unique_lock<std::mutex> lock(s->mu);
            s->cv_work.wait_for(lock, std::chrono::microseconds(200),
                                [&] { return s->stop || !s->pending.empty(); });
            if (s->stop) break;
        }
        {
            std::lock_guard<std::mutex> lock(s->mu);
            if (s->stop) {
                if (running) {
                    cp_batch_interrupt(s->batch);
                    int a = 0, d = 0;
                    cp_batch_wait(s->batch, &a, &d);
                    running = false;
                }
                for (auto& r : ready) r->status = CP_ERR_CANCELLED;
                for (auto& r : s->lane_q) {
                    s->inflight_bytes -= r->footprint;
                    r->status = CP_ERR_CANCELLED;
                    complete(s, r);
                }
                s->lane_q.clear();
                s->cv_done.notify_all();
                break;
            }
        }
    }
}

}  // namespace

extern "C" {

CP_API void cp_server_opts_default(cp_server_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->device = 0;
    o->hbm_reserve = 0.05;
    o->max_inflight = 1024;
    o->trip_quantum = 0;
    cp_batch_opts_default(&o->batch);
    o->fp64_lanes = 8;
}

CP_API int cp_server_create(const cp_server_opts* opts, cp_server** out) {
    if (!out) return CP_ERR_INVALID;
    *out = nullptr;
    cp_server_opts o;
    cp_server_opts_default(&o);
    if (opts) o = *opts;
    if (o.max_inflight <= 0 || !(o.hbm_reserve >= 0.0 && o.hbm_reserve < 1.0) || o.fp64_lanes < 0 ||
        o.fp64_lanes > 64)
        return CP_ERR_INVALID;
    if (o.max_inflight > o.batch.max_instances) o.max_inflight = o.batch.max_instances;
    cp_server* s = new (std::nothrow) cp_server();
    if (!s) return CP_ERR_NOMEM;
    s->o = o;
    int rc = cp_context_create(o.device, &s->ctx_run);
    if (rc == CP_OK) rc = cp_context_create(o.device, &s->ctx_setup);
    if (rc == CP_OK) rc = cp_context_create(o.device, &s->ctx_out);
    if (rc == CP_OK) rc = cp_batch_create(s->ctx_run, &o.batch, &s->batch);
    for (int k = 0; rc == CP_OK && k < o.fp64_lanes; ++k) {
        cp_context* c = nullptr;
        rc = cp_context_create(o.device, &c);
        if (rc == CP_OK) s->lane_ctx.push_back(c);
    }
    s->lane_cur.assign(s->lane_ctx.size(), nullptr);
    {
        const char* e = std::getenv("CUPLAST_LANE_PRIORITY");
        int least = 0, greatest = 0;
        if (rc == CP_OK && !(e && e[0] == '0') && cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess &&
            greatest < least) {
            for (cp_context* c : s->lane_ctx) {
                s->lane_own.push_back(c->stream);
                std::vector<cudaStream_t> v;
                for (int p = greatest; p <= least && rc == CP_OK; ++p) {  // greatest priority first
                    cudaStream_t st = nullptr;
                    if (cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, p) != cudaSuccess) rc = CP_ERR_CUDA;
                    else v.push_back(st);
                }
                s->lane_streams.push_back(v);
            }
            s->lane_level.assign(s->lane_ctx.size(), -1);
        }
    }
    if (rc == CP_OK) {
        size_t f = 0, t = 0;
        if (cudaMemGetInfo(&f, &t) != cudaSuccess) rc = CP_ERR_CUDA;
        s->total_mem = t;
    }
    if (rc != CP_OK) {
        release_lane_streams(s);
        for (cp_context* c : s->lane_ctx) cp_context_destroy(c);
        if (s->batch) cp_batch_destroy(s->batch);
        if (s->ctx_out) cp_context_destroy(s->ctx_out);
        if (s->ctx_setup) cp_context_destroy(s->ctx_setup);
        if (s->ctx_run) cp_context_destroy(s->ctx_run);
        delete s;
        return rc;
    }
    try {
        std::lock_guard<std::mutex> lock(g_live_mu);
        if (!g_atexit_registered) g_atexit_registered = std::atexit(stop_all_at_exit) == 0;
        s->th = std::thread(scheduler, s);
        for (int k = 0; k < (int)s->lane_ctx.size(); ++k) s->lanes.emplace_back(lane, s, k);
        g_live.push_back(s);
    } catch (...) {
        {
            std::lock_guard<std::mutex> lock(s->mu);
            s->stop = true;
        }
        s->cv_work.notify_all();
        s->cv_lane.notify_all();
        if (s->th.joinable()) s->th.join();
        for (auto& t : s->lanes)
            if (t.joinable()) t.join();
        release_lane_streams(s);
        for (cp_context* c : s->lane_ctx) cp_context_destroy(c);
        cp_batch_destroy(s->batch);
        cp_context_destroy(s->ctx_out);
        cp_context_destroy(s->ctx_setup);
        cp_context_destroy(s->ctx_run);
        delete s;
        return CP_ERR_NOMEM;
    }
    *out = s;
    return CP_OK;
}

CP_API int cp_server_destroy(cp_server* s) {
    if (!s) return CP_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lock(g_live_mu);
        g_live.erase(std::remove(g_live.begin(), g_live.end(), s), g_live.end());
    }
    stop_thread(s);
    cp_batch_destroy(s->batch);  // releases the instances it still owned
    std::lock_guard<std::mutex> lock(s->mu);
    for (auto& kv : s->by_id) {
        ReqP r = kv.second;
        if (r->inst) cp_instance_destroy(r->inst);
        r->inst = nullptr;
        if (!r->done) {
            r->status = CP_ERR_CANCELLED;
            r->done = true;
        }
    }
    s->cv_done.notify_all();
    release_lane_streams(s);
    for (cp_context* c : s->lane_ctx) cp_context_destroy(c);
    cp_context_destroy(s->ctx_out);
    cp_context_destroy(s->ctx_setup);
    cp_context_destroy(s->ctx_run);
    delete s;
    return CP_OK;
}

CP_API int cp_server_submit(cp_server* s, const cp_mesh_view* mv, const cp_material* mat, const double* rp,
                            const unsigned char* mask, const double* uv, const cp_solve_opts* opts, long long* id) {
    if (!s || !mv || !mat || !rp || !mask || !opts || !id) return CP_ERR_INVALID;
    if (opts->precision != CP_PREC_MIXED && opts->precision != CP_PREC_FP64 && opts->precision != CP_PREC_FLOAT_BOOST)
        return CP_ERR_INVALID;
    if (is_lane_request(*opts) && s->o.fp64_lanes == 0) return CP_ERR_UNSUPPORTED;
    if (mv->node_count <= 0 || !mv->node_xy || mv->count3 < 0 || mv->count4 < 0 || mv->count8 < 0 ||
        (long long)mv->count3 + mv->count4 + mv->count8 <= 0 || (mv->count3 && !mv->elem3) ||
        (mv->count4 && !mv->elem4) || (mv->count8 && !mv->elem8))
        return CP_ERR_INVALID;
    auto r = std::make_shared<Request>();
    const size_t n2 = 2 * (size_t)mv->node_count;
    try {
        r->nn = mv->node_count;
        r->c3 = mv->count3;
        r->c4 = mv->count4;
        r->c8 = mv->count8;
        r->xy.assign(mv->node_xy, mv->node_xy + n2);
        if (mv->count3) r->e3.assign(mv->elem3, mv->elem3 + 3 * (size_t)mv->count3);
        if (mv->count4) r->e4.assign(mv->elem4, mv->elem4 + 4 * (size_t)mv->count4);
        if (mv->count8) r->e8.assign(mv->elem8, mv->elem8 + 8 * (size_t)mv->count8);
        r->rp.assign(rp, rp + n2);
        r->mask.assign(mask, mask + n2);
        if (uv) {
            r->uv.assign(uv, uv + n2);
            r->has_uv = true;
        }
    } catch (const std::bad_alloc&) {
        return CP_ERR_NOMEM;
    }
    r->mat = *mat;
    r->opts = *opts;
    int rc = cp_instance_footprint(mv, opts->precision, &r->footprint);
    if (rc != CP_OK) return rc;
    if (opts->precond == 2) {  // the multigrid hierarchy, built at the request's first solve
        // directed neighbour links: at most n_en (n_en - 1) per element
        const size_t links = 6 * (size_t)mv->count3 + 12 * (size_t)mv->count4 + 56 * (size_t)mv->count8;
        r->footprint += cp::mg_footprint((size_t)mv->node_count, (size_t)mv->node_count + links);
    }
    const size_t reserve = (size_t)(s->o.hbm_reserve * (double)s->total_mem);
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stop) return CP_ERR_CANCELLED;
    if (r->footprint + reserve > s->total_mem || (s->o.max_bytes && r->footprint > s->o.max_bytes)) {
        s->st.rejected += 1;
        return CP_ERR_NOMEM;
    }
    r->id = s->next_id++;
    r->t_submit = Clock::now();
    s->pending.push_back(r);
    s->by_id[r->id] = r;
    s->st.submitted += 1;
    *id = r->id;
    s->cv_work.notify_all();
    return CP_OK;
}

CP_API int cp_server_wait(cp_server* s, long long id, double timeout_s, cp_instance** inst, cp_solve_report* report,
                          double* latency_s) {
    if (!s) return CP_ERR_INVALID;
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->by_id.find(id);
    if (it == s->by_id.end()) return CP_ERR_INVALID;
    ReqP r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_s < 0) {
        s->cv_done.wait(lock, ready);
    } else if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), ready)) {
        return CP_ERR_BUSY;
    }
    s->by_id.erase(id);
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    if (report) *report = r->rep;
    if (r->status != CP_OK) {
        if (report) report->status = r->status;
        if (inst) *inst = nullptr;
        return r->status;
    }
    if (inst) {
        *inst = r->inst;
    } else {
        cp_instance_destroy(r->inst);
    }
    r->inst = nullptr;
    return CP_OK;
}

CP_API int cp_server_get_stats(cp_server* s, cp_server_stats* out) {
    if (!s || !out) return CP_ERR_INVALID;
    std::lock_guard<std::mutex> lock(s->mu);
    cp_server_stats st = s->st;
    st.inflight = (long long)s->inflight.size();
    st.pending = (long long)s->pending.size();
    *out = st;
    return CP_OK;
}

}  // extern "C"
