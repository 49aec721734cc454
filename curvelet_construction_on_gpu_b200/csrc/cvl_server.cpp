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
    bool done = false;
    int status = CVL_OK;
    std::string err;
    cvl_result *res = nullptr;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct cvl_server {
    cvl_server_cfg cfg{};
    cvl_params params{};
    std::vector<cvl_engine *> engines;
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
            lat_ms.push_back(ms_between(r->t_submit, Clock::now()));
            lat_edges.push_back(r->n);
            lat_ids.push_back(r->id);
        } else {
            ++failed;
        }
    }

    void worker(int w);

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
    cvl_batch *batch = nullptr;
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
                if (admitted + r->charge > cfg.mem_budget_bytes) break;
                lanes[l].pop_front();
                queue_ms += ms_between(r->t_submit, Clock::now());
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
        std::vector<cvl_result *> outs(take.size(), nullptr);
        std::vector<int> st(take.size(), rc);
        std::vector<std::string> errs(take.size(), err);
        if (rc == CVL_OK) {
            for (size_t m = 0; m < take.size(); ++m) {
                st[m] = cvl_batch_result_take_map(br, (int32_t)m, &outs[m]);
                if (st[m] != CVL_OK) errs[m] = cvl_last_error();
            }
        }
        if (br) cvl_batch_result_free(br);
        const Clock::time_point t3 = Clock::now();
        {
            std::lock_guard<std::mutex> lk(mu);
            upload_ms += ms_between(t0, t1);
            run_ms += ms_between(t1, t2);
            device_ms += dev_ms;
            result_ms += ms_between(t2, t3);
            for (size_t m = 0; m < take.size(); ++m) {
                host.put(take[m]->edges);
                take[m]->edges = nullptr;
                finish(take[m], st[m], errs[m], outs[m]);
            }
            if (lane_now == 0) --small_running;
        }
        cv_done.notify_all();
        cv_work.notify_all();  // budget freed
        cv_yield.notify_all();
    }
    if (batch) cvl_batch_free(batch);
}

extern "C" {

void cvl_server_cfg_default(cvl_server_cfg *c) {
    if (!c) return;
    c->device = 0;
    c->workers = 4;
    c->mem_budget_bytes = (size_t)40 << 30;
    c->admit_bytes_per_edge = 2048;
    c->max_batch_edges = 2 << 20;
    c->large_map_edges = 1000000;
    c->host_reserve_bytes = (size_t)2 << 30;
    c->small_takes_large = 0;
    c->large_workers = 0;
    c->large_yield_ms = 10;
    c->device_reserve_bytes = 0;
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
    if (c.mem_budget_bytes == 0 || c.admit_bytes_per_edge == 0 || c.max_batch_edges <= 0 || c.large_map_edges <= 0)
        return cvl_fail(CVL_EINVAL, "budget, admission charge and batch sizes must be > 0");
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
        // device memory for the largest launch the worker will fold (admission's model of
        // the footprint), mapped now so that the stream never waits on a memory mapping
        size_t dev_reserve = c.device_reserve_bytes;
        if (!dev_reserve)
            dev_reserve = std::min((size_t)c.max_batch_edges * c.admit_bytes_per_edge,
                                   c.mem_budget_bytes / (size_t)c.workers);
        int rr = cvl_engine_reserve_device(e, dev_reserve);
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
    const size_t charge = (size_t)num_edges * s->cfg.admit_bytes_per_edge;
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
    for (cvl_engine *e : s->engines) cvl_engine_destroy(e);
    delete s;
}

}  // extern "C"
