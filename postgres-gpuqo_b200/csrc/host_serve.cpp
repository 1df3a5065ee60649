// host_serve.cpp - continuous-batching planner service.
//
// Requests (gpuqo_b200_server_submit) are planned concurrently: each runs its
// planner (BFS relabel, IDP2 / UnionDP or one exact DP) on a worker thread,
// at most max_inflight at a time; further requests queue for a slot.  Every
// exact DP a planner needs is handed to one scheduler thread, which runs
// whatever sub-problems are pending as one level-synchronous wave on the
// batched engine (admitted by dense-memo bytes), then wakes their planners.
// Sub-problems that arrive while a wave is on the GPU join the next wave, so
// the device stays busy with the union of all in-flight queries' work.
// Sub-problems outside the batched kernel's scope (plain DPsub, very large
// biconnected blocks) run one by one on the single-query engine.
//
// With gpuqo_b200_devices other than 1 the service has one such scheduler
// (a lane) per device; a request is given to the lane with the fewest
// requests in flight and all its exact DPs run there.
//
// Each plan is the one gpuqo_run returns for the same query and settings: the
// sub-problems are identical, only the way they share the GPU differs.
//
// This service is for standalone planning processes; inside a Postgres
// backend (single-threaded, palloc not thread-safe) use gpuqo_run.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "dp_engine.h"
#include "gpuqo_b200.h"
#include "host_idp.h"
#include "host_info.h"

extern "C" int gpuqo_idp_n_iters;
extern "C" int gpuqo_idp_type;
extern "C" bool gpuqo_dpsub_bicc_enable;
extern "C" bool gpuqo_dpsub_ccc_enable;

extern "C" int gpuqo_b200_server_batch_window_us;

namespace gqb {

void set_error(int code, const std::string &msg);
int exact_dp(const HostInfo &info, DpMode mode, std::vector<TreeNode> &nodes, std::string &err);

using Clock = std::chrono::steady_clock;

struct SubTask {
    std::vector<uint32_t> blob;
    DpMode mode;
    int n;
    std::vector<TreeNode> nodes;
    int rc = 0;
    std::string err;
    bool done = false;
};

struct Request {
    uint64_t id;
    int lane = 0;                      // the device lane that runs its exact DPs
    PlannerHandle *planner = nullptr;
    Clock::time_point t_submit, t_done;
    int rc = 0;
    std::string err;
    bool started = false, done = false;
    std::thread th;
};

// One device of the service (gpuqo_b200_devices): its scheduler thread runs
// the pending sub-problems of the requests given to this device.
struct DevLane {
    int device = 0;
    std::deque<SubTask *> pending;
    std::condition_variable cv;
    std::thread th;
    int load = 0;                      // requests given to this lane and not finished
    int active = 0;                    // of those, planners running (not queued for a slot)
};

// the lane for a new request: the one with the fewest requests in flight
// (the lowest index on ties)
static int pick_lane(const std::vector<std::unique_ptr<DevLane>> &lanes) {
    int best = 0;
    for (int i = 1; i < (int)lanes.size(); i++)
        if (lanes[(size_t)i]->load < lanes[(size_t)best]->load) best = i;
    return best;
}

class Server {
public:
    int max_inflight = 16;
    uint64_t wave_bytes = 32ull << 30;
    bool ccc = true;

    std::mutex mu;
    std::condition_variable cv_sub, cv_req;
    std::vector<std::unique_ptr<DevLane>> lanes;
    bool stopping = false;

    std::map<uint64_t, std::unique_ptr<Request>> reqs;
    std::deque<Request *> waiting;   // submitted, no slot yet
    int running = 0;
    uint64_t next_id = 1;

    // counters
    uint64_t completed = 0, waves = 0, wave_items = 0, singles = 0;
    double device_ms = 0.0, busy_ms = 0.0, starved_ms = 0.0;

    int start(std::string &err) {
        std::vector<int> devs;
        if (int rc = batch_devices(devs, err)) return rc;
        for (int d : devs) {
            lanes.emplace_back(new DevLane());
            lanes.back()->device = d;
        }
        for (auto &ln : lanes) {
            DevLane *l = ln.get();
            l->th = std::thread([this, l] { scheduler(*l); });
        }
        return 0;
    }

    // exact DP of one sub-problem, through its lane's scheduler (called by planners)
    int solve(int lane, const HostInfo &h, DpMode mode, std::vector<TreeNode> &nodes, std::string &err) {
        // sub-problems on the sparse memo (32 to 63 relations, or fewer under
        // gpuqo_b200_sparse_from_rels) run directly on the request's thread
        if (use_sparse_memo(h.n, mode)) {
            cudaSetDevice(lanes[(size_t)lane]->device);
            return exact_dp(h, mode, nodes, err);
        }
        SubTask t;
        t.blob = build_blob(h);
        apply_dpsub_csg(t.blob, mode);
        t.mode = mode;
        t.n = h.n;
        {
            std::unique_lock<std::mutex> lk(mu);
            lanes[(size_t)lane]->pending.push_back(&t);
            lanes[(size_t)lane]->cv.notify_one();
            cv_sub.wait(lk, [&] { return t.done; });
        }
        if (t.rc) {
            err = t.err;
            return t.rc;
        }
        nodes = std::move(t.nodes);
        return 0;
    }

    void scheduler(DevLane &ln) {
        cudaSetDevice(ln.device);
        std::deque<SubTask *> &pending = ln.pending;
        for (;;) {
            std::vector<SubTask *> tasks;
            {
                std::unique_lock<std::mutex> lk(mu);
                const bool open = ln.load > 0;
                const Clock::time_point t_wait = Clock::now();
                ln.cv.wait(lk, [&] { return stopping || !pending.empty(); });
                if (open) starved_ms += std::chrono::duration<double, std::milli>(Clock::now() - t_wait).count();
                if (stopping && pending.empty()) return;
                // batching window: planners of this lane that are between two
                // sub-problems (running, nothing pending) usually submit their
                // next one within tens of microseconds; a wave costs about the
                // same device time for a few sub-problems as for many, so wait
                // up to gpuqo_b200_server_batch_window_us for them
                if (gpuqo_b200_server_batch_window_us > 0) {
                    const Clock::time_point until =
                        Clock::now() + std::chrono::microseconds(gpuqo_b200_server_batch_window_us);
                    ln.cv.wait_until(lk, until, [&] { return stopping || (int)pending.size() >= ln.active; });
                }
                // admit pending sub-problems while the wave's memory fits
                uint64_t bytes = 0;
                while (!pending.empty()) {
                    SubTask *t = pending.front();
                    uint64_t b = batch_query_bytes(t->n);
                    if (!tasks.empty() && bytes + b > wave_bytes) break;
                    pending.pop_front();
                    tasks.push_back(t);
                    bytes += b;
                }
            }
            const Clock::time_point t_busy = Clock::now();
            std::vector<SubTask *> batch, one;
            for (SubTask *t : tasks)
                if (t->mode == kModeMpdp && t->n <= 30 && batch_eligible(t->blob)) batch.push_back(t);
                else one.push_back(t);
            if (!batch.empty()) {
                std::vector<const std::vector<uint32_t> *> blobs;
                for (SubTask *t : batch) blobs.push_back(&t->blob);
                std::vector<std::vector<TreeNode>> out;
                std::vector<double> wave_ms;
                EngineStats st;
                std::string err;
                int rc = engine_run_batch(blobs, wave_bytes, out, st, wave_ms, err);
                std::lock_guard<std::mutex> lk(mu);
                waves += wave_ms.size();
                wave_items += batch.size();
                device_ms += st.device_ms;
                for (size_t i = 0; i < batch.size(); i++) {
                    batch[i]->rc = rc;
                    batch[i]->err = err;
                    if (!rc) batch[i]->nodes = std::move(out[i]);
                    batch[i]->done = true;
                }
                cv_sub.notify_all();
            }
            for (SubTask *t : one) {
                EngineStats st;
                std::string err;
                std::vector<TreeNode> nodes;
                int rc = engine_run(t->blob, t->n, t->mode, ccc, false, nodes, st, err);
                std::lock_guard<std::mutex> lk(mu);
                singles++;
                device_ms += st.device_ms;
                t->rc = rc;
                t->err = err;
                t->nodes = std::move(nodes);
                t->done = true;
                cv_sub.notify_all();
            }
            std::lock_guard<std::mutex> lk(mu);
            busy_ms += std::chrono::duration<double, std::milli>(Clock::now() - t_busy).count();
        }
    }

    // caller holds mu
    void launch(Request *r) {
        r->started = true;
        running++;
        lanes[(size_t)r->lane]->active++;
        r->th = std::thread([this, r] {
            cudaSetDevice(lanes[(size_t)r->lane]->device);
            std::string err;
            int rc = planner_run(r->planner, err);
            std::lock_guard<std::mutex> lk(mu);
            r->rc = rc;
            r->err = err;
            r->t_done = Clock::now();
            r->done = true;
            running--;
            lanes[(size_t)r->lane]->load--;
            lanes[(size_t)r->lane]->active--;
            lanes[(size_t)r->lane]->cv.notify_one();   // one planner fewer to wait for
            completed++;
            if (!waiting.empty()) {
                Request *nx = waiting.front();
                waiting.pop_front();
                launch(nx);
            }
            cv_req.notify_all();
        });
    }

    int submit(int algorithm, const GpuqoPlannerInfoC *info, uint64_t *ticket, std::string &err) {
        auto r = std::make_unique<Request>();
        r->t_submit = Clock::now();
        {
            std::lock_guard<std::mutex> lk(mu);
            r->lane = pick_lane(lanes);
            lanes[(size_t)r->lane]->load++;
        }
        const int lane = r->lane;
        SubSolver solver = [this, lane](const HostInfo &h, DpMode m, std::vector<TreeNode> &nodes, std::string &e) {
            return solve(lane, h, m, nodes, e);
        };
        r->planner = planner_new(algorithm, info, gpuqo_idp_n_iters, gpuqo_idp_type, solver, err);
        std::lock_guard<std::mutex> lk(mu);
        if (!r->planner) {
            lanes[(size_t)lane]->load--;
            return GPUQO_B200_ERR_ARGS;
        }
        r->id = next_id++;
        *ticket = r->id;
        Request *raw = r.get();
        reqs[r->id] = std::move(r);
        if (running < max_inflight) launch(raw);
        else waiting.push_back(raw);
        return 0;
    }

    // the request stops before its next exact DP (planner_cancel) and its
    // wait returns GPUQO_B200_ERR_CANCELLED, unless it has already finished;
    // the other requests, and the waves it shared with them, are unaffected
    int cancel(uint64_t ticket, std::string &err) {
        std::lock_guard<std::mutex> lk(mu);
        auto it = reqs.find(ticket);
        if (it == reqs.end()) {
            err = "unknown ticket";
            return GPUQO_B200_ERR_ARGS;
        }
        planner_cancel(it->second->planner);
        return 0;
    }

    int wait(uint64_t ticket, QueryTreeC **out, double *latency_ms, std::string &err) {
        Request *r;
        {
            std::unique_lock<std::mutex> lk(mu);
            auto it = reqs.find(ticket);
            if (it == reqs.end()) {
                err = "unknown ticket";
                return GPUQO_B200_ERR_ARGS;
            }
            r = it->second.get();
            cv_req.wait(lk, [&] { return r->done; });
        }
        r->th.join();
        // take the request out of the table before its planner is freed, so
        // that a concurrent cancel finds no planner to touch
        std::unique_ptr<Request> own;
        {
            std::lock_guard<std::mutex> lk(mu);
            auto it = reqs.find(ticket);
            own = std::move(it->second);
            reqs.erase(it);
        }
        int rc = own->rc;
        if (out) *out = rc ? nullptr : planner_result(own->planner);
        if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(own->t_done - own->t_submit).count();
        if (rc) err = own->err;
        planner_free(own->planner);
        return rc;
    }

    void stop() {
        // finish outstanding requests (they still need the scheduler), then
        // stop the scheduler
        std::vector<uint64_t> tickets;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (auto &kv : reqs) tickets.push_back(kv.first);
        }
        for (uint64_t t : tickets) {
            std::string e;
            wait(t, nullptr, nullptr, e);
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            stopping = true;
            for (auto &ln : lanes) ln->cv.notify_all();
        }
        for (auto &ln : lanes)
            if (ln->th.joinable()) ln->th.join();
    }
};

static std::mutex g_srv_mu;
static std::unique_ptr<Server> g_server;

}  // namespace gqb

using namespace gqb;

extern "C" int gpuqo_b200_server_start(int max_inflight, int wave_memory_mb) {
    std::lock_guard<std::mutex> lk(g_srv_mu);
    if (g_server) return GPUQO_B200_ERR_ARGS;
    auto s = std::make_unique<Server>();
    s->max_inflight = max_inflight > 0 ? max_inflight : 16;
    s->wave_bytes = (uint64_t)std::max(wave_memory_mb, 64) << 20;
    s->ccc = gpuqo_dpsub_ccc_enable;
    std::string err;
    if (int rc = s->start(err)) {
        set_error(rc, err);
        return rc;
    }
    g_server = std::move(s);
    return GPUQO_B200_OK;
}

extern "C" int gpuqo_b200_server_submit(int gpuqo_algorithm, GpuqoPlannerInfoC *info, uint64_t *ticket) {
    if (!g_server || !info || !ticket) return GPUQO_B200_ERR_ARGS;
    std::string err;
    int rc = g_server->submit(gpuqo_algorithm, info, ticket, err);
    if (rc) set_error(rc, err);
    return rc;
}

extern "C" int gpuqo_b200_server_wait(uint64_t ticket, QueryTreeC **out, double *latency_ms) {
    if (!g_server) return GPUQO_B200_ERR_ARGS;
    std::string err;
    int rc = g_server->wait(ticket, out, latency_ms, err);
    if (rc) set_error(rc, err);
    return rc;
}

extern "C" int gpuqo_b200_server_cancel(uint64_t ticket) {
    if (!g_server) return GPUQO_B200_ERR_ARGS;
    std::string err;
    int rc = g_server->cancel(ticket, err);
    if (rc) set_error(rc, err);
    return rc;
}

extern "C" int gpuqo_b200_server_stats(GpuqoB200ServerStats *out) {
    if (!g_server || !out) return GPUQO_B200_ERR_ARGS;
    std::lock_guard<std::mutex> lk(g_server->mu);
    out->completed = g_server->completed;
    out->waves = g_server->waves;
    out->batched_subproblems = g_server->wave_items;
    out->single_subproblems = g_server->singles;
    out->device_ms = g_server->device_ms;
    out->busy_ms = g_server->busy_ms;
    out->starved_ms = g_server->starved_ms;
    return GPUQO_B200_OK;
}

extern "C" int gpuqo_b200_server_stop(void) {
    std::lock_guard<std::mutex> lk(g_srv_mu);
    if (!g_server) return GPUQO_B200_ERR_ARGS;
    g_server->stop();
    g_server.reset();
    return GPUQO_B200_OK;
}
