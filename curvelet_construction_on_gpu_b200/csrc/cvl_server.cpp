// cvl_server.cpp -- continuous batching over libcvl engines (cvl_server_* in
// include/cvl.h).
//
// Requests are queued on the host. Each worker (one engine: its own stream and
// workspace on the server's device) runs a loop in its own host thread:
//   1. Take waiting requests from one lane, in arrival order, while they fit the
//      launch (max_batch_edges) and the admission budget.
//   2. Refill the worker's device batch straight from the requests'
//      page-locked blocks. The buffer is grow-only, so there is no cudaFree and
//      no device-wide synchronisation.
//   3. Run the whole path over the ragged batch.
//   4. Copy each map's rows into its own page-locked result.
//   5. Release the budget.
// Workers run concurrently, so one batch's copies and kernels overlap another's.
// Small and large maps have separate lanes, so a small map never waits behind a
// 4K map in the same launch.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cvl.h"
#include "cvl_internal.h"
#include "cvl_pinned.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    double *edges = nullptr;  // page-locked, from the server's arena
    int32_t n = 0, sz = 4;
    size_t charge = 0;
    int lane = 0;
    Clock::time_point t_submit;
    cvl_request_times times{};  // filled as the request goes through
    bool done = false;
    int status = CVL_OK;
    std::string err;
    cvl_result *res = nullptr;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

// maps folded into one launch at most (the reserved workspace's per-map statistics)
constexpr int32_t MAX_MAPS_PER_LAUNCH = 4096;

struct cvl_server {
    cvl_server_cfg cfg{};
    cvl_params params{};
    cvl_tuning tune[CVL_TUNING_BUCKETS];  // the workers' tuning (the footprint's bundle chunk)
    std::vector<cvl_engine *> engines;
    std::vector<cvl_batch *> wbatch;  // each worker's device batch, reserved at creation
    size_t reserved = 0;              // device workspace reserved by the workers
    std::vector<std::thread> threads;
    cvl::PinnedArena host;

    std::mutex mu;
    std::condition_variable cv_work;  // workers: requests queued or stop
    std::condition_variable cv_done;  // waiters: a request finished
    std::condition_variable cv_yield; // large launches waiting for the small lane to drain
    int small_running = 0;            // small-lane launches on the device
    std::deque<Request *> lanes[2];   // 0 small, 1 large
    std::unordered_map<uint64_t, Request *> reqs;
    std::deque<uint64_t> finished;    // ids in completion order, not handed out yet
    uint64_t next_id = 1;
    size_t admitted = 0;
    bool stop = false;

    uint64_t submitted = 0, completed = 0, failed = 0, in_flight = 0, launches = 0, edges_completed = 0;
    double upload_ms = 0, run_ms = 0, device_ms = 0, result_ms = 0, queue_ms = 0;
    std::vector<double> lat_ms;
    std::vector<int64_t> lat_edges;
    std::vector<uint64_t> lat_ids;
    std::vector<cvl_request_times> lat_times;

    // the lane a worker serves first (the last large_workers workers prefer large maps when there are several)
    int preferred_lane(int w) const { return (cfg.workers >= 2 && w >= cfg.workers - cfg.large_workers) ? 1 : 0; }

    // lane whose head request fits the remaining budget, preferred lane first; -1 if none
    int lane_to_take(int w) const {
        const int pref = preferred_lane(w);
        const int nlanes = (pref == 0 && !cfg.small_takes_large && cfg.workers >= 2) ? 1 : 2;
        for (int k = 0; k < nlanes; ++k) {
            const int l = k == 0 ? pref : 1 - pref;
            if (!lanes[l].empty() && admitted + lanes[l].front()->charge <= cfg.mem_budget_bytes) return l;
        }
        return -1;
    }

    void finish(Request *r, int status, const std::string &err, cvl_result *res) {
        // called with mu held
        r->done = true;
        r->status = status;
        r->err = err;
        r->res = res;
        admitted -= r->charge;
        --in_flight;
        finished.push_back(r->id);
        if (status == CVL_OK) {
            ++completed;
            edges_completed += (uint64_t)r->n;
            const double total = ms_between(r->t_submit, Clock::now());
            lat_ms.push_back(total);
            lat_edges.push_back(r->n);
            lat_ids.push_back(r->id);
            r->times.id = r->id;
            r->times.edges = r->n;
            r->times.total_ms = total;
            lat_times.push_back(r->times);
        } else {
            ++failed;
        }
    }

    void worker(int w);

    // The launch shape of n edges (sz values each, maps maps) at the configured
    // pairs and curvelets per edge.
    cvl_workspace_shape shape_of(int64_t n, int32_t sz, int32_t maps) const {
        cvl_workspace_shape sh;
        sh.num_edges = n;
        sh.num_pairs = (int64_t)std::ceil((double)n * cfg.pairs_per_edge);
        sh.num_curvelets = (int64_t)std::ceil((double)n * cfg.curvelets_per_edge);
        sh.num_maps = maps;
        sh.edge_data_sz = sz;
        return sh;
    }

    // A request's admission charge: its workspace footprint (a launch of the map
    // alone, less the bundle chunk that each worker holds once), or the per-edge charge.
    size_t charge_of(int64_t n, int32_t sz) const {
        if (cfg.admit_bytes_per_edge) return (size_t)n * cfg.admit_bytes_per_edge;
        const cvl_workspace_shape sh = shape_of(n, sz, 1);
        size_t total = 0, chunk = 0;
        if (cvl_workspace_bytes_tuned(tune, &sh, &params, &total, &chunk) != CVL_OK) return (size_t)-1;
        return total - chunk;
    }

    // The largest map of at most cap edges whose charge fits the budget (0 if none).
    int64_t largest_admissible(int64_t cap) const {
        int64_t lo = 0, hi = cap;
        while (lo < hi) {
            const int64_t mid = lo + (hi - lo + 1) / 2;
            if (charge_of(mid, 4) <= cfg.mem_budget_bytes) lo = mid; else hi = mid - 1;
        }
        return lo;
    }

    // Engine hook of a worker running a large launch, called between its chunks:
    // while small-lane work is queued or running, hold back (large_yield_ms at most), so
    // that a small map does not share the SMs with a large map's chunks. Only
    // when the server is not backlogged: with requests piling up, the GPU must
    // not idle and the large launch goes on.
    static constexpr size_t YIELD_MAX_QUEUED = 4;
    static void yield_to_small(void *ctx) {
        cvl_server *s = (cvl_server *)ctx;
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_yield.wait_for(lk, std::chrono::milliseconds(s->cfg.large_yield_ms), [&] {
            const size_t queued = s->lanes[0].size() + s->lanes[1].size();
            return s->stop || queued > YIELD_MAX_QUEUED || (s->small_running == 0 && s->lanes[0].empty());
        });
    }
};

void cvl_server::worker(int w) {
    cudaSetDevice(cfg.device);
    cvl_engine *e = engines[w];
    cvl_batch *batch = wbatch[w];
    std::vector<Request *> take;
    std::vector<int32_t> counts;
    std::vector<const double *> parts;
    int lane_now = 0;
    while (true) {
        take.clear();
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stop || lane_to_take(w) >= 0; });
            if (stop) break;
            const int l = lane_to_take(w);
            lane_now = l;
            int64_t sum = 0;
            while (!lanes[l].empty()) {
                Request *r = lanes[l].front();
                if (!take.empty() && sum + r->n > cfg.max_batch_edges) break;
                if ((int32_t)take.size() >= MAX_MAPS_PER_LAUNCH) break;
                if (admitted + r->charge > cfg.mem_budget_bytes) break;
                lanes[l].pop_front();
                r->times.queue_ms = ms_between(r->t_submit, Clock::now());
                r->times.worker = w;
                queue_ms += r->times.queue_ms;
                admitted += r->charge;
                ++in_flight;
                take.push_back(r);
                sum += r->n;
            }
            ++launches;
            if (lane_now == 0) ++small_running;
        }
        cv_yield.notify_all();
        // a large launch yields to small ones between its chunks (with another worker to run them)
        cvl_engine_set_yield(e, (lane_now == 1 && cfg.workers >= 2 && cfg.large_yield_ms > 0)
                                    ? &cvl_server::yield_to_small : nullptr, this);
        // one edge_data_sz per launch: a request with another width goes alone
        size_t cut = 1;
        while (cut < take.size() && take[cut]->sz == take[0]->sz) ++cut;
        if (cut < take.size()) {
            std::lock_guard<std::mutex> lk(mu);
            for (size_t k = take.size(); k-- > cut;) {
                Request *r = take[k];
                admitted -= r->charge;
                --in_flight;
                lanes[r->lane].push_front(r);
            }
            take.resize(cut);
            cv_work.notify_all();
        }
        const int32_t sz = take[0]->sz;
        counts.clear();
        parts.clear();
        for (Request *r : take) {
            counts.push_back(r->n);
            parts.push_back(r->edges);
        }
        int rc = CVL_OK;
        std::string err;
        cvl_batch_result *br = nullptr;
        const Clock::time_point t0 = Clock::now();
        if (!batch) {
            // the first launch makes the worker's batch; later ones refill it
            rc = cvl_batch_upload(e, parts[0], counts.data(), 1, sz, &batch);
        }
        if (rc == CVL_OK) rc = cvl_batch_refill_parts(batch, parts.data(), counts.data(), (int32_t)counts.size(), sz);
        const Clock::time_point t1 = Clock::now();
        if (rc == CVL_OK) rc = cvl_batch_run(e, batch, &params, &br);
        if (rc != CVL_OK) err = cvl_last_error();
        const Clock::time_point t2 = Clock::now();
        double dev_ms = 0.0;
        if (br) {
            cvl_batch_stats bst;
            if (cvl_batch_result_stats(br, &bst) == CVL_OK) dev_ms = bst.device_ms;
        }
        const double t_up = ms_between(t0, t1), t_run = ms_between(t1, t2);
        {
            std::lock_guard<std::mutex> lk(mu);
            upload_ms += t_up;
            run_ms += t_run;
            device_ms += dev_ms;
        }
        // each map's rows to its own result; a request is finished as soon as its
        // rows are copied (not at the end of the launch's copies)
        for (size_t m = 0; m < take.size(); ++m) {
            cvl_result *out = nullptr;
            int stm = rc;
            std::string errm = err;
            if (rc == CVL_OK) {
                stm = cvl_batch_result_take_map(br, (int32_t)m, &out);
                if (stm != CVL_OK) errm = cvl_last_error();
            }
            const Clock::time_point tm = Clock::now();
            {
                std::lock_guard<std::mutex> lk(mu);
                Request *r = take[m];
                r->times.upload_ms = t_up;
                r->times.run_ms = t_run;
                r->times.result_ms = ms_between(t2, tm);
                r->times.launch_maps = (int32_t)take.size();
                host.put(r->edges);
                r->edges = nullptr;
                finish(r, stm, errm, out);
                if (m + 1 == take.size()) {
                    result_ms += ms_between(t2, tm);
                    if (lane_now == 0) --small_running;
                }
            }
            cv_done.notify_all();
        }
        if (br) cvl_batch_result_free(br);
        cv_done.notify_all();
        cv_work.notify_all();  // budget freed
        cv_yield.notify_all();
    }
}

extern "C" {

void cvl_server_cfg_default(cvl_server_cfg *c) {
    if (!c) return;
    c->device = 0;
    c->workers = 4;
    c->mem_budget_bytes = (size_t)40 << 30;
    c->max_batch_edges = 2 << 20;
    c->large_map_edges = 1000000;
    c->host_reserve_bytes = (size_t)2 << 30;
    c->small_takes_large = 0;
    c->large_workers = 0;
    c->large_yield_ms = 10;
    c->device_reserve_bytes = 0;
    c->admit_bytes_per_edge = 0;
    c->max_map_edges = 4 << 20;
    c->pairs_per_edge = 40.0;
    c->curvelets_per_edge = 8.0;
}

int cvl_server_create(const cvl_server_cfg *cfg, const cvl_params *p, cvl_server **out) {
    if (!out || !p) return cvl_fail(CVL_EINVAL, "out/params is NULL");
    *out = nullptr;
    cvl_server_cfg c;
    cvl_server_cfg_default(&c);
    if (cfg) c = *cfg;
    if (c.workers < 1 || c.workers > 16) return cvl_fail(CVL_EINVAL, "workers must be in [1, 16]");
    if (c.large_yield_ms < 0 || c.large_yield_ms > 1000) return cvl_fail(CVL_EINVAL, "large_yield_ms must be in [0, 1000]");
    if (c.large_workers == 0) c.large_workers = std::max(1, c.workers / 2);
    if (c.workers >= 2 && c.large_workers >= c.workers) c.large_workers = c.workers - 1;
    if (c.large_workers < 1) return cvl_fail(CVL_EINVAL, "large_workers must be 0 (automatic) or in [1, workers - 1]");
    if (c.mem_budget_bytes == 0 || c.max_batch_edges <= 0 || c.large_map_edges <= 0 || c.max_map_edges <= 0)
        return cvl_fail(CVL_EINVAL, "budget, batch sizes and max_map_edges must be > 0");
    if (!(c.pairs_per_edge >= 0.0 && c.pairs_per_edge <= 1024.0) ||
        !(c.curvelets_per_edge >= 0.0 && c.curvelets_per_edge <= 1024.0))
        return cvl_fail(CVL_EINVAL, "pairs_per_edge and curvelets_per_edge must be in [0, 1024]");
    cvl_server *s = new cvl_server();
    s->cfg = c;
    s->params = *p;
    for (int w = 0; w < c.workers; ++w) {
        cvl_engine_cfg ec;
        cvl_engine_cfg_default(&ec);
        ec.device = c.device;
        // small-lane workers first on the device (the lowest number is the highest priority)
        const bool small_lane = !(c.workers >= 2 && w >= c.workers - c.large_workers);
        ec.stream_priority = small_lane ? -1000 : 0;
        cvl_engine *e = nullptr;
        const int rc = cvl_engine_create(&ec, &e);
        if (rc != CVL_OK) {
            const std::string msg = cvl_last_error();
            for (cvl_engine *x : s->engines) cvl_engine_destroy(x);
            delete s;
            return cvl_fail(rc, msg);
        }
        s->engines.push_back(e);
        if (w == 0) {
            for (int b = 0; b < CVL_TUNING_BUCKETS; ++b) cvl_engine_get_tuning(e, b, &s->tune[b]);
        }
        // The workspace of the largest launch the worker's lane takes, allocated now, so
        // that the stream never waits on a memory mapping: max_batch_edges folded maps
        // for a small-lane worker, the largest map for a large-lane one (which also takes
        // small maps when its lane is empty); no more than the budget admits.
        const bool takes_large = !small_lane || c.workers < 2 || c.small_takes_large;
        const int64_t lane_edges = takes_large ? std::max(c.max_map_edges, c.max_batch_edges) : c.max_batch_edges;
        const int64_t n_res = std::max<int64_t>(s->largest_admissible(std::min<int64_t>(lane_edges, 0x7fffffffLL)), 1);
        const cvl_workspace_shape sh = s->shape_of(n_res, 4, MAX_MAPS_PER_LAUNCH);
        size_t ws_total = 0;
        int rr = cvl_engine_workspace_bytes(e, &sh, p, &ws_total, nullptr);
        if (rr == CVL_OK) rr = cvl_engine_reserve_workspace(e, &sh, p);
        cvl_batch *wb = nullptr;
        if (rr == CVL_OK) rr = cvl_batch_create_reserved(e, n_res, MAX_MAPS_PER_LAUNCH, 4, &wb);
        s->wbatch.push_back(wb);
        s->reserved += ws_total;
        if (rr == CVL_OK && c.device_reserve_bytes) rr = cvl_engine_reserve_device(e, c.device_reserve_bytes);
        if (rr == CVL_OK) rr = cvl_engine_reserve_host(e, c.host_reserve_bytes);
        if (rr != CVL_OK) {
            const std::string msg = cvl_last_error();
            for (cvl_engine *x : s->engines) cvl_engine_destroy(x);
            delete s;
            return cvl_fail(rr, msg);
        }
    }
    if (c.host_reserve_bytes && !s->host.reserve(c.host_reserve_bytes)) {
        for (cvl_engine *x : s->engines) cvl_engine_destroy(x);
        delete s;
        return cvl_fail(CVL_ENOMEM, "page-locked host memory could not be reserved");
    }
    for (int w = 0; w < c.workers; ++w) s->threads.emplace_back(&cvl_server::worker, s, w);
    *out = s;
    return CVL_OK;
}

int cvl_server_submit(cvl_server *s, const double *edges, int32_t num_edges, int32_t edge_data_sz, uint64_t *id) {
    const Clock::time_point t_call = Clock::now();  // latency counts the copy below
    if (!s || !edges || !id) return cvl_fail(CVL_EINVAL, "server/edges/id is NULL");
    if (num_edges <= 0 || edge_data_sz < 4) return cvl_fail(CVL_EINVAL, "num_edges <= 0 or edge_data_sz < 4");
    if (num_edges > s->cfg.max_map_edges)
        return cvl_fail(CVL_ENOMEM, "a map of " + std::to_string(num_edges) + " edges is larger than max_map_edges (" +
                                        std::to_string(s->cfg.max_map_edges) + ")");
    const size_t charge = s->charge_of(num_edges, edge_data_sz);
    if (charge > s->cfg.mem_budget_bytes)
        return cvl_fail(CVL_ENOMEM, "a map of " + std::to_string(num_edges) + " edges needs " + std::to_string(charge) +
                                        " bytes of admission budget; the budget is " +
                                        std::to_string(s->cfg.mem_budget_bytes));
    Request *r = new Request();
    const size_t nval = (size_t)num_edges * edge_data_sz;
    r->edges = (double *)s->host.get(sizeof(double) * nval);
    if (!r->edges) {
        delete r;
        return cvl_fail(CVL_ENOMEM, "page-locked request buffer could not be allocated");
    }
    std::memcpy(r->edges, edges, sizeof(double) * nval);
    r->n = num_edges;
    r->sz = edge_data_sz;
    r->charge = charge;
    r->lane = (num_edges >= s->cfg.large_map_edges) ? 1 : 0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            s->host.put(r->edges);
            delete r;
            return cvl_fail(CVL_EINVAL, "server is stopping");
        }
        r->id = s->next_id++;
        r->t_submit = t_call;
        s->reqs[r->id] = r;
        s->lanes[r->lane].push_back(r);
        ++s->submitted;
        *id = r->id;
    }
    s->cv_work.notify_all();
    return CVL_OK;
}

namespace {

// hands out a finished request's result and forgets the request (mu held)
int hand_out(cvl_server *s, std::unordered_map<uint64_t, Request *>::iterator it, cvl_result **out) {
    Request *r = it->second;
    s->reqs.erase(it);
    auto f = std::find(s->finished.begin(), s->finished.end(), r->id);
    if (f != s->finished.end()) s->finished.erase(f);
    const int st = r->status;
    const std::string err = r->err;
    *out = r->res;
    delete r;
    if (st != CVL_OK) return cvl_fail(st, err);
    return CVL_OK;
}

}  // namespace

int cvl_server_poll(cvl_server *s, uint64_t id, cvl_result **out) {
    if (!s || !out) return cvl_fail(CVL_EINVAL, "server/out is NULL");
    *out = nullptr;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return cvl_fail(CVL_EINVAL, "unknown request id (or its result was handed out)");
    if (!it->second->done) return cvl_fail(CVL_EAGAIN, "request not finished");
    return hand_out(s, it, out);
}

int cvl_server_wait(cvl_server *s, uint64_t id, int64_t timeout_us, cvl_result **out) {
    if (!s || !out) return cvl_fail(CVL_EINVAL, "server/out is NULL");
    *out = nullptr;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return cvl_fail(CVL_EINVAL, "unknown request id (or its result was handed out)");
    Request *r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_us < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), ready)) {
        return cvl_fail(CVL_ETIMEDOUT, "request not finished within the timeout");
    }
    return hand_out(s, s->reqs.find(id), out);
}

int cvl_server_next(cvl_server *s, int64_t timeout_us, uint64_t *id, cvl_result **out) {
    if (!s || !id || !out) return cvl_fail(CVL_EINVAL, "server/id/out is NULL");
    *out = nullptr;
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [&] { return !s->finished.empty() || s->reqs.empty(); };
    if (timeout_us < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), ready)) {
        return cvl_fail(CVL_ETIMEDOUT, "no request finished within the timeout");
    }
    if (s->finished.empty()) return cvl_fail(CVL_EAGAIN, "no request is queued or running");
    *id = s->finished.front();
    return hand_out(s, s->reqs.find(*id), out);
}

int cvl_server_stats_get(cvl_server *s, cvl_server_stats *out) {
    if (!s || !out) return cvl_fail(CVL_EINVAL, "server/out is NULL");
    std::vector<double> l;
    cvl_server_stats st{};
    {
        std::lock_guard<std::mutex> lk(s->mu);
        st.submitted = s->submitted;
        st.completed = s->completed;
        st.failed = s->failed;
        st.queued = s->lanes[0].size() + s->lanes[1].size();
        st.in_flight = s->in_flight;
        st.launches = s->launches;
        st.edges_completed = s->edges_completed;
        st.admitted_bytes = s->admitted;
        st.upload_ms = s->upload_ms;
        st.run_ms = s->run_ms;
        st.device_ms = s->device_ms;
        st.result_ms = s->result_ms;
        st.queue_ms = s->queue_ms;
        st.reserved_bytes = s->reserved;
        l = s->lat_ms;
    }
    st.host_grows = s->host.grows();
    st.host_grow_ms = s->host.grow_ms();
    for (cvl_engine *e : s->engines) {
        uint64_t dg = 0, hg = 0;
        double dms = 0, hms = 0;
        cvl_engine_growth(e, &dg, &dms, &hg, &hms);
        st.device_grows += dg;
        st.device_grow_ms += dms;
        st.host_grows += hg;
        st.host_grow_ms += hms;
    }
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) {  // nearest rank
            size_t k = (size_t)std::ceil(q * (double)l.size());
            return l[std::min(l.size() - 1, k ? k - 1 : 0)];
        };
        st.p50_ms = pct(0.50);
        st.p95_ms = pct(0.95);
        st.p99_ms = pct(0.99);
        st.max_ms = l.back();
    }
    *out = st;
    return CVL_OK;
}

int64_t cvl_server_latencies(cvl_server *s, double *ms, int64_t *edges, uint64_t *ids, int64_t cap) {
    if (!s || cap < 0 || (cap > 0 && (!ms || !edges))) return cvl_fail(CVL_EINVAL, "invalid arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    const int64_t n = std::min<int64_t>(cap, (int64_t)s->lat_ms.size());
    for (int64_t k = 0; k < n; ++k) {
        ms[k] = s->lat_ms[k];
        edges[k] = s->lat_edges[k];
        if (ids) ids[k] = s->lat_ids[k];
    }
    return n;
}

int64_t cvl_server_request_times(cvl_server *s, cvl_request_times *out, int64_t cap) {
    if (!s || cap < 0 || (cap > 0 && !out)) return cvl_fail(CVL_EINVAL, "invalid arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    const int64_t n = std::min<int64_t>(cap, (int64_t)s->lat_times.size());
    for (int64_t k = 0; k < n; ++k) out[k] = s->lat_times[k];
    return n;
}

void cvl_server_destroy(cvl_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (auto &q : s->lanes) {
            for (Request *r : q) {
                s->host.put(r->edges);
                r->edges = nullptr;
                r->done = true;
                r->status = CVL_EINVAL;
                r->err = "server stopped before the request was admitted";
                ++s->failed;
            }
            q.clear();
        }
    }
    s->cv_work.notify_all();
    s->cv_yield.notify_all();
    for (std::thread &t : s->threads) t.join();
    s->cv_done.notify_all();
    for (auto &kv : s->reqs) {
        if (kv.second->res) cvl_result_free(kv.second->res);
        delete kv.second;
    }
    for (cvl_engine *e : s->engines) cvl_engine_destroy(e);  // frees each engine's batches too
    delete s;
}

}  // extern "C"
