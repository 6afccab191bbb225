// Serving loop: partial-aggregation requests from many executor tasks arrive
// as they please; each names one live query whose table stays resident in
// HBM. A dispatcher thread admits queued requests in arrival order as soon
// as a device slot is free and the HBM budget (resident tables + in-flight
// staging) allows, so requests that arrive while others run overlap on the
// device (continuous batching, not a queue drained one at a time). Each query
// keeps at most two requests in flight (its handle's two staging sets); other
// queries proceed meanwhile on their own streams. Completion is stamped by a
// host callback enqueued behind the request's work; latency = submit ->
// completion. No reference analogue: VecRuntime runs inside Spark tasks.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "runtime.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    int qid = -1;
    vr_batch batch{};
    std::vector<vr_column> cols;
    int64_t bytes = 0;
    Clock::time_point t_submit;
    Clock::time_point t_admit;
    Clock::time_point t_done;
    int state = 0;  // 0 queued, 1 running, 2 done
    int status = VR_OK;
    bool queued_wait = false;  // not admitted at its first scan
};

struct Query {
    vr_agg* h = nullptr;
    int in_flight = 0;
    int64_t table_bytes = 0;
    bool closed = false;
};

}  // namespace

struct vr_srv {
    vr_srv_config cfg{};
    std::mutex mu;
    std::condition_variable cv;       // dispatcher wake-ups
    std::condition_variable done_cv;  // waiters
    std::deque<std::shared_ptr<Request>> queue;
    std::map<uint64_t, std::shared_ptr<Request>> tickets;
    std::vector<Query> queries;
    std::vector<double> latencies_ms;
    std::vector<double> waits_ms;     // submit -> admit
    std::vector<double> services_ms;  // admit -> done
    int in_flight = 0;
    int64_t in_flight_bytes = 0;
    int64_t table_bytes = 0;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread dispatcher;
    vr_srv_stats st{};
};

namespace {

struct CallbackArg {
    vr_srv* s;
    std::shared_ptr<Request> r;
};

void CUDART_CB on_done(void* p) {
    CallbackArg* a = static_cast<CallbackArg*>(p);
    vr_srv* s = a->s;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        Request& r = *a->r;
        r.t_done = Clock::now();
        r.state = 2;
        s->in_flight--;
        s->in_flight_bytes -= r.bytes;
        s->queries[r.qid].in_flight--;
        double ms = std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count();
        s->latencies_ms.push_back(ms);
        s->waits_ms.push_back(std::chrono::duration<double, std::milli>(r.t_admit - r.t_submit).count());
        s->services_ms.push_back(std::chrono::duration<double, std::milli>(r.t_done - r.t_admit).count());
        s->st.completed++;
        s->st.rows += r.batch.num_rows;
        s->st.hbm_in_use = s->table_bytes + s->in_flight_bytes;
    }
    s->cv.notify_all();
    s->done_cv.notify_all();
    delete a;
}

// A query's resident device bytes: its table (which grows as groups arrive)
// plus both staging sets and deferred-row lists.
int64_t query_bytes(const vr_agg* h) {
    int64_t tb = h->table_slots * h->plan.prog.sw * 8;
    for (const vr::StageSlot& sl : h->slot) tb += (int64_t)sl.dev_cap + sl.deferred_cap * 16;
    return tb;
}

int64_t batch_bytes(const vr_agg* h, const vr_batch& b) {
    int64_t n = b.num_rows, bytes = 0;
    const vr::Program& P = h->plan.prog;
    for (int c = 0; c < P.num_cols; ++c) {
        int w = P.col_width[c];
        bytes += w ? n * w : (n + 7) / 8;
        bytes += (n + 7) / 8;
    }
    return bytes + (n + 7) / 8;
}

void dispatch_loop(vr_srv* s) {
    cudaSetDevice(s->cfg.device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        bool launched = false;
        for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
            auto r = *it;
            Query& q = s->queries[r->qid];
            if (s->in_flight >= s->cfg.slots) {
                for (auto& w : s->queue) w->queued_wait = true;
                break;
            }
            if (q.in_flight >= 2) {  // the handle's two staging sets are busy
                r->queued_wait = true;
                continue;
            }
            if (s->table_bytes + s->in_flight_bytes + r->bytes > s->cfg.hbm_cap_bytes && s->in_flight > 0) {
                r->queued_wait = true;
                continue;
            }
            s->queue.erase(it);
            r->state = 1;
            r->t_admit = Clock::now();
            s->in_flight++;
            s->st.max_in_flight = std::max<int64_t>(s->st.max_in_flight, s->in_flight);
            s->in_flight_bytes += r->bytes;
            q.in_flight++;
            s->st.hbm_in_use = s->table_bytes + s->in_flight_bytes;
            s->st.hbm_peak = std::max(s->st.hbm_peak, s->st.hbm_in_use);
            if (r->queued_wait) s->st.queued++; else s->st.admitted_immediately++;
            vr_agg* h = q.h;
            lk.unlock();
            int rc = vr_agg_update(h, &r->batch);
            const int64_t now = query_bytes(h);  // the update may have grown the table
            CallbackArg* arg = new CallbackArg{s, r};
            const bool ok = rc == VR_OK && cudaLaunchHostFunc(h->stream, on_done, arg) == cudaSuccess;
            lk.lock();
            // the query list may have grown (and moved) while the lock was released
            Query& qn = s->queries[r->qid];
            if (ok) {
                s->table_bytes += now - qn.table_bytes;
                qn.table_bytes = now;
                s->st.hbm_peak = std::max(s->st.hbm_peak, s->table_bytes + s->in_flight_bytes);
            } else {
                delete arg;
                r->status = rc == VR_OK ? VR_ERR_CUDA : rc;
                r->state = 2;
                r->t_done = Clock::now();
                s->in_flight--;
                s->in_flight_bytes -= r->bytes;
                qn.in_flight--;
                s->done_cv.notify_all();
            }
            launched = true;
            break;  // restart the scan: state changed
        }
        if (!launched) s->cv.wait_for(lk, std::chrono::milliseconds(2));
    }
}

double percentile(std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    double idx = p * (v.size() - 1);
    size_t lo = (size_t)idx;
    size_t hi = std::min(lo + 1, v.size() - 1);
    double f = idx - lo;
    return v[lo] * (1 - f) + v[hi] * f;
}

}  // namespace

extern "C" {

int vr_srv_create(const vr_srv_config* cfg, vr_srv** out) {
    if (!cfg || !out) return VR_ERR_INVALID;
    vr_srv* s = new vr_srv();
    s->cfg = *cfg;
    if (s->cfg.slots <= 0) s->cfg.slots = 32;
    if (s->cfg.hbm_cap_bytes <= 0) s->cfg.hbm_cap_bytes = 120ll << 30;
    if (cudaSetDevice(s->cfg.device) != cudaSuccess) {
        delete s;
        return VR_ERR_CUDA;
    }
    s->dispatcher = std::thread(dispatch_loop, s);
    *out = s;
    return VR_OK;
}

int vr_srv_open_query(vr_srv* s, const vr_agg_spec* spec, int32_t* query_id) {
    if (!s || !spec || !query_id) return VR_ERR_INVALID;
    vr_agg* h = nullptr;
    int rc = vr_agg_create(spec, &h);
    if (rc != VR_OK) return rc;
    // requests arrive from host memory at up to max_batch_rows rows: size the
    // staging now, so the dispatcher never frees and reallocates it (cudaFree
    // would stall every query's pipeline)
    if ((rc = vr::agg_reserve(h, spec->max_batch_rows)) != VR_OK) {
        vr_agg_destroy(h);
        return rc;
    }
    const int64_t tb = query_bytes(h);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->table_bytes + tb > s->cfg.hbm_cap_bytes) {
        vr_agg_destroy(h);
        s->st.rejected++;
        return VR_ERR_ADMISSION;
    }
    Query q;
    q.h = h;
    q.table_bytes = tb;
    s->table_bytes += tb;
    s->queries.push_back(q);
    *query_id = (int32_t)s->queries.size() - 1;
    return VR_OK;
}

int vr_srv_submit(vr_srv* s, int32_t qid, const vr_batch* batch, uint64_t* ticket) {
    if (!s || !batch || !ticket || batch->location != VR_HOST) return VR_ERR_INVALID;
    auto r = std::make_shared<Request>();
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (qid < 0 || qid >= (int)s->queries.size() || s->queries[qid].closed) return VR_ERR_INVALID;
        vr_agg* h = s->queries[qid].h;
        r->qid = qid;
        r->batch = *batch;
        r->cols.assign(batch->columns, batch->columns + h->spec.num_columns);
        r->batch.columns = r->cols.data();
        r->bytes = batch_bytes(h, *batch);
        if (s->table_bytes + r->bytes > s->cfg.hbm_cap_bytes) {
            s->st.rejected++;
            return VR_ERR_ADMISSION;
        }
        r->ticket = s->next_ticket++;
        s->tickets[r->ticket] = r;
        s->queue.push_back(r);
        s->st.submitted++;
        *ticket = r->ticket;
    }
    s->cv.notify_all();
    return VR_OK;
}

int vr_srv_wait(vr_srv* s, uint64_t ticket, double* latency_ms) {
    if (!s) return VR_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return VR_ERR_INVALID;
    auto r = it->second;
    s->done_cv.wait(lk, [&] { return r->state == 2; });
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    s->tickets.erase(ticket);
    return r->status;
}

int vr_srv_drain(vr_srv* s) {
    if (!s) return VR_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    s->done_cv.wait(lk, [&] { return s->queue.empty() && s->in_flight == 0; });
    return VR_OK;
}

int vr_srv_query_handle(vr_srv* s, int32_t qid, vr_agg** h) {
    if (!s || !h) return VR_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    if (qid < 0 || qid >= (int)s->queries.size()) return VR_ERR_INVALID;
    s->done_cv.wait(lk, [&] {
        if (s->queries[qid].in_flight) return false;
        for (auto& r : s->queue)
            if (r->qid == qid) return false;
        return true;
    });
    *h = s->queries[qid].h;
    lk.unlock();
    return vr_agg_sync(*h);
}

int vr_srv_close_query(vr_srv* s, int32_t qid) {
    vr_agg* h = nullptr;
    int rc = vr_srv_query_handle(s, qid, &h);
    if (rc != VR_OK && rc != VR_ERR_STATE && !h) return rc;
    std::lock_guard<std::mutex> lk(s->mu);
    Query& q = s->queries[qid];
    if (!q.closed) {
        q.closed = true;
        s->table_bytes -= q.table_bytes;
        vr_agg_destroy(q.h);
        q.h = nullptr;
    }
    return VR_OK;
}

int vr_srv_get_stats(vr_srv* s, vr_srv_stats* st) {
    if (!s || !st) return VR_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    *st = s->st;
    st->p50_ms = percentile(s->latencies_ms, 0.50);
    st->p99_ms = percentile(s->latencies_ms, 0.99);
    st->p99_wait_ms = percentile(s->waits_ms, 0.99);
    st->p99_service_ms = percentile(s->services_ms, 0.99);
    double mx = 0, sum = 0;
    for (double v : s->latencies_ms) {
        mx = std::max(mx, v);
        sum += v;
    }
    st->max_ms = mx;
    st->mean_ms = s->latencies_ms.empty() ? 0 : sum / s->latencies_ms.size();
    return VR_OK;
}

void vr_srv_destroy(vr_srv* s) {
    if (!s) return;
    vr_srv_drain(s);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    for (auto& q : s->queries)
        if (q.h) vr_agg_destroy(q.h);
    delete s;
}

}  // extern "C"
