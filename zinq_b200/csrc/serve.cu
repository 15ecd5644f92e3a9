// serve.cu -- a job server for streams of independent propagation requests.
//
// Requests are validated and copied at submission.  Worker threads (one CUDA stream per job)
// admit them in arrival order while their estimated device memory fits the budget and the
// device's measured free memory.  A worker advances its jobs in launches of `stream_steps`
// steps (zqd_job_step): 1-D single-solve requests that share a kernel shape (precision, states,
// grid points) form one group advanced by one launch of the resident line kernel, every member
// from its own step; between launches finished or cancelled members leave and waiting requests
// of the same shape join (continuous batching).  Other requests run on their own.  After every
// launch the new observable rows of each job are posted as events (zqd_server_poll); completion,
// failure and cancellation are events too, and zqd_server_wait hands the result over.
// The reference has no serving layer: this is the request loop around its quantum_dynamics.run.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "internal.h"
#include "job.h"
#include "line_kernel.cuh"

namespace {

using Clock = std::chrono::steady_clock;

enum class State { Queued, Running, Done };

struct Request {
    uint64_t ticket = 0;
    zqd::Opts o;
    size_t est = 0;         // estimated device bytes while it runs
    uint64_t group_key = 0; // 0: runs alone; else requests with equal keys share launches
    Clock::time_point t0, t1;
    State state = State::Queued;
    int status = ZQD_OK;
    std::string error;
    zqd_result* result = nullptr;
    std::atomic<bool> cancel{false};
    zqd_job* job = nullptr; // while running (owned by the worker)
    ~Request() {
        if (result) zqd_result_destroy(result);
    }
};
using Req = std::shared_ptr<Request>;

struct Event {
    uint64_t ticket = 0;
    int kind = ZQD_EVENT_ROWS, status = ZQD_OK;
    uint32_t solve = 0, first_row = 0, nrows = 0, width = 0;
    int solve_finished = 0;
    std::vector<double> rows;
};

// Upper bound of a job's device allocations (tables, wavefunction copies, history, scratch).
size_t estimate_bytes(const zqd::Opts& o) {
    size_t N = 1;
    for (uint32_t i = 0; i < o.ndim; ++i) N *= o.npoint;
    const size_t S = (size_t)o.pot_ns, c = o.precision == ZQD_FP32_MIXED ? 8 : 16, nsolve = o.imag_nstate ? o.imag_nstate : 1;
    const size_t nsym = S * (S + 1) / 2;
    size_t b = (4 + nsolve) * S * N * c;                     // psi, phi, psi0, initial state, relaxed states
    b += nsym * N * 16 + N * 16 + 2 * S * S * N * 8 + N * 8; // R, kinetic phase, V and U, cap weights
    b += nsolve * ((size_t)o.iterations + 1) * (size_t)zqd::RowLayout{(int)o.ndim, (int)S}.width() * 8;
    if (o.write_mask & ZQD_WRITE_WAVEFUNCTION) b += nsolve * ((size_t)o.iterations + 1) * S * N * c;
    b += N / 4 * 8 * 48 + (1u << 20);                        // partial sums, small tables, slack
    return b;
}

uint64_t group_key(const zqd::Opts& o) {
    if (o.ndim != 1 || o.imag_nstate > 1) return 0;
    return 1 + ((uint64_t)o.npoint << 8) + ((uint64_t)o.pot_ns << 2) + ((uint64_t)o.precision << 1);
}

// every finite entry of the recorded columns (the others are NaN by design) of new rows
bool rows_finite(const zqd_obs_rows& r, int d, int S, uint32_t wmask) {
    const zqd::RowLayout L{d, S};
    for (uint32_t k = 0; k < r.nrows; ++k) {
        const double* row = r.rows + (size_t)k * r.width;
        if ((wmask & ZQD_WRITE_NORM) && !std::isfinite(row[L.norm()])) return false;
        if (wmask & ZQD_WRITE_POPULATION)
            for (int s = 0; s < S; ++s)
                if (!std::isfinite(row[L.pop() + s])) return false;
    }
    return true;
}

} // namespace

struct zqd_server {
    int device = 0;
    size_t budget = 0, in_use = 0, peak = 0;
    uint32_t max_batch = 16, stream_steps = 256, max_events = 65536;
    bool stream_rows = true;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req> queue;
    std::unordered_map<uint64_t, Req> live;
    std::deque<Event> events;
    std::vector<Event> polled; // the rows handed out by the last zqd_server_poll
    uint64_t next_ticket = 1;
    bool stop = false;
    zqd_server_stats stats{};
    std::vector<std::thread> workers;

    bool fits(const Request& q) const; // under mu
    void work();
    void run_active(std::vector<Req> group);
    void post(Event&& e);                           // under mu
    void finish(const Req& q, int status, const std::string& err, zqd_result* res); // takes mu
    void stream(const Req& q);
};

bool zqd_server::fits(const Request& q) const {
    if (in_use + q.est > budget) return false;
    if (in_use == 0) return true; // nothing of ours to wait for: the allocation decides
    return q.est + q.est / 8 <= zqd::device_free_bytes();
}

void zqd_server::post(Event&& e) {
    if (!stream_rows && e.kind == ZQD_EVENT_ROWS) return;
    if (events.size() >= max_events) { // a consumer that stopped polling: drop the oldest row events
        auto it = std::find_if(events.begin(), events.end(), [](const Event& x) { return x.kind == ZQD_EVENT_ROWS; });
        if (it != events.end()) {
            events.erase(it);
            ++stats.dropped_events;
        } else if (e.kind == ZQD_EVENT_ROWS) {
            ++stats.dropped_events;
            return;
        }
    }
    events.push_back(std::move(e));
}

void zqd_server::finish(const Req& q, int status, const std::string& err, zqd_result* res) {
    std::lock_guard<std::mutex> lk(mu);
    q->status = status;
    q->error = err;
    q->result = res;
    q->t1 = Clock::now();
    q->state = State::Done;
    in_use -= q->est;
    ++stats.completed;
    if (status == ZQD_ERR_CANCELLED) ++stats.cancelled;
    else if (status) ++stats.failed;
    Event e;
    e.ticket = q->ticket;
    e.kind = status == ZQD_OK ? ZQD_EVENT_DONE : status == ZQD_ERR_CANCELLED ? ZQD_EVENT_CANCELLED : ZQD_EVENT_FAILED;
    e.status = status;
    post(std::move(e));
    cv_done.notify_all();
    cv_work.notify_all();
}

// the job's observable rows recorded since the last call, as events
void zqd_server::stream(const Req& q) {
    for (;;) {
        zqd_obs_rows r{};
        if (zqd_job_observables(q->job, &r) != ZQD_OK || r.nrows == 0) return;
        if (!rows_finite(r, (int)q->o.ndim, q->o.pot_ns, q->o.write_mask)) throw ZQD_ERR_NUMERIC;
        Event e;
        e.ticket = q->ticket;
        e.solve = r.solve;
        e.first_row = r.first_row;
        e.nrows = r.nrows;
        e.width = r.width;
        e.solve_finished = r.solve_finished;
        if (stream_rows) e.rows.assign(r.rows, r.rows + (size_t)r.nrows * r.width);
        std::lock_guard<std::mutex> lk(mu);
        post(std::move(e));
    }
}

// Advances `group` (one request, or 1-D requests of one shape) launch by launch until every
// member has left; waiting requests of the same shape join between launches.
void zqd_server::run_active(std::vector<Req> group) {
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        for (const Req& q : group) finish(q, ZQD_ERR_DEVICE, "cudaStreamCreateWithFlags failed", nullptr);
        return;
    }
    const uint64_t key = group.front()->group_key;
    auto create = [&](const Req& q) -> bool {
        zqd::Opts o = q->o;
        const int rc = zqd::job_create_opts(std::move(o), &q->job);
        if (rc) {
            finish(q, rc, zqd::last_error(), nullptr);
            q->job = nullptr;
            return false;
        }
        q->job->nd_use_graph = false;
        return true;
    };
    std::vector<Req> active;
    for (const Req& q : group)
        if (create(q)) active.push_back(q);
    const uint32_t chunk = stream_steps ? stream_steps : UINT32_MAX;
    while (!active.empty()) {
        // members whose cancellation was requested leave before the launch
        for (auto it = active.begin(); it != active.end();) {
            if ((*it)->cancel.load()) {
                zqd_job_destroy((*it)->job);
                (*it)->job = nullptr;
                finish(*it, ZQD_ERR_CANCELLED, "CANCELLED", nullptr);
                it = active.erase(it);
            } else {
                ++it;
            }
        }
        if (active.empty()) break;
        // one launch per resolved precision (ZQD_PRECISION_AUTO requests resolve at creation)
        std::vector<zqd_job*> sub[2];
        std::vector<Req> subq[2];
        for (const Req& q : active) {
            const int g = key && q->job->d == 1 ? (q->job->fp32 ? 1 : 0) : -1;
            if (g < 0) {
                const int rc = zqd_job_step(q->job, chunk);
                if (rc) q->status = rc, q->error = zqd::last_error();
            } else {
                sub[g].push_back(q->job);
                subq[g].push_back(q);
            }
        }
        for (int g = 0; g < 2; ++g) {
            if (sub[g].empty()) continue;
            const int rc = zqd::step_line_group(sub[g], chunk, st);
            {
                std::lock_guard<std::mutex> lk(mu);
                ++stats.grouped_launches;
                stats.grouped_jobs += sub[g].size();
            }
            if (rc)
                for (const Req& q : subq[g]) q->status = rc, q->error = zqd::last_error();
        }
        // stream the new rows; members that ended (or failed) leave
        for (auto it = active.begin(); it != active.end();) {
            const Req& q = *it;
            int rc = q->status;
            int finished = 0;
            if (!rc) {
                try {
                    stream(q);
                } catch (int e) {
                    rc = e;
                    q->error = "NON-FINITE OBSERVABLE (the wavefunction norm or a population is NaN or Inf)";
                }
                zqd_job_progress(q->job, nullptr, nullptr, &finished);
            }
            if (!rc && !finished) {
                ++it;
                continue;
            }
            zqd_result* res = nullptr;
            if (!rc && (rc = zqd_job_result(q->job, &res))) q->error = zqd::last_error();
            if (!rc) { // the final observables (always computed) must be finite
                for (uint32_t s = 0; s < zqd_result_nsolve(res) && !rc; ++s) {
                    zqd_observables ob{};
                    zqd_result_final(res, s, &ob);
                    if (!std::isfinite(ob.norm)) {
                        rc = ZQD_ERR_NUMERIC;
                        q->error = "NON-FINITE OBSERVABLE (the wavefunction norm is NaN or Inf)";
                    }
                }
                if (rc) {
                    zqd_result_destroy(res);
                    res = nullptr;
                }
            }
            zqd_job_destroy(q->job);
            q->job = nullptr;
            finish(q, rc, rc ? q->error : std::string(), res);
            it = active.erase(it);
        }
        // continuous batching: waiting requests of this shape take the free slots
        if (key) {
            std::vector<Req> joined;
            {
                std::lock_guard<std::mutex> lk(mu);
                for (auto it = queue.begin(); it != queue.end() && active.size() + joined.size() < max_batch;) {
                    if ((*it)->group_key == key && fits(**it)) {
                        in_use += (*it)->est;
                        peak = std::max(peak, in_use);
                        stats.peak_device_bytes = peak;
                        (*it)->state = State::Running;
                        joined.push_back(*it);
                        ++stats.joined_jobs;
                        it = queue.erase(it);
                    } else {
                        ++it;
                    }
                }
            }
            for (const Req& q : joined)
                if (create(q)) active.push_back(q);
        }
    }
    cudaStreamDestroy(st);
}

void zqd_server::work() {
    cudaSetDevice(device);
    for (;;) {
        std::vector<Req> batch;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return (stop && queue.empty()) || (!queue.empty() && fits(*queue.front())); });
            if (queue.empty()) return;
            // the head, then waiting requests of its shape while they fit (arrival order)
            Req head = queue.front();
            queue.pop_front();
            batch.push_back(head);
            in_use += head->est;
            if (head->group_key)
                for (auto it = queue.begin(); it != queue.end() && batch.size() < max_batch;) {
                    if ((*it)->group_key == head->group_key && fits(**it)) {
                        in_use += (*it)->est;
                        batch.push_back(*it);
                        it = queue.erase(it);
                    } else {
                        ++it;
                    }
                }
            for (const Req& q : batch) q->state = State::Running;
            peak = std::max(peak, in_use);
            stats.peak_device_bytes = peak;
            if (!queue.empty()) cv_work.notify_one();
        }
        run_active(std::move(batch));
    }
}

extern "C" void zqd_server_config_init(zqd_server_config* cfg) {
    if (!cfg) return;
    *cfg = zqd_server_config{};
    cfg->struct_size = sizeof(zqd_server_config);
    cfg->workers = 4;
    cfg->max_batch = 16;
    cfg->stream_steps = 256;
    cfg->stream_rows = 1;
    cfg->max_events = 65536;
}

extern "C" int zqd_server_create(const zqd_server_config* cfg, zqd_server** out) {
    if (!cfg || !out) return zqd::fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    *out = nullptr;
    if (cfg->struct_size != sizeof(zqd_server_config))
        return zqd::fail(ZQD_ERR_INVALID_INPUT, "zqd_server_config.struct_size does not match this library");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return zqd::fail(ZQD_ERR_NO_DEVICE, "no CUDA device");
    std::unique_ptr<zqd_server> S(new (std::nothrow) zqd_server());
    if (!S) return zqd::fail(ZQD_ERR_OUT_OF_MEMORY, "host allocation failed");
    ZQD_CUDA(cudaGetDevice(&S->device));
    const size_t free_b = zqd::device_free_bytes();
    S->budget = cfg->device_budget_bytes ? (size_t)cfg->device_budget_bytes : free_b / 10 * 9;
    S->max_batch = std::max(1u, cfg->max_batch ? cfg->max_batch : 16u);
    S->stream_steps = cfg->stream_steps;
    S->stream_rows = cfg->stream_rows != 0;
    S->max_events = std::max(1u, cfg->max_events ? cfg->max_events : 65536u);
    S->stats.device_budget_bytes = S->budget;
    const uint32_t nw = std::max(1u, cfg->workers ? cfg->workers : 4u);
    for (uint32_t i = 0; i < nw; ++i) S->workers.emplace_back([s = S.get()] { s->work(); });
    *out = S.release();
    return ZQD_OK;
}

extern "C" int zqd_server_submit(zqd_server* S, const zqd_options* opt, uint64_t* ticket) {
    if (!S || !ticket) return zqd::fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    auto q = std::make_shared<Request>();
    int rc = zqd::copy_options(opt, q->o);
    if (rc) return rc;
    if ((rc = zqd::validate(q->o))) return rc;
    q->est = estimate_bytes(q->o);
    q->group_key = group_key(q->o);
    std::lock_guard<std::mutex> lk(S->mu);
    if (q->est > S->budget) return zqd::fail(ZQD_ERR_DEVICE_OOM, "REQUEST NEEDS MORE DEVICE MEMORY THAN THE SERVER BUDGET");
    if (S->stop) return zqd::fail(ZQD_ERR_CANCELLED, "SERVER IS SHUTTING DOWN");
    q->ticket = S->next_ticket++;
    q->t0 = Clock::now();
    *ticket = q->ticket;
    S->live[q->ticket] = q;
    S->queue.push_back(q);
    ++S->stats.submitted;
    S->cv_work.notify_one();
    return ZQD_OK;
}

extern "C" int zqd_server_cancel(zqd_server* S, uint64_t ticket) {
    if (!S) return zqd::fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    Req q;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->live.find(ticket);
        if (it == S->live.end()) return zqd::fail(ZQD_ERR_NOT_FOUND, "UNKNOWN TICKET");
        q = it->second;
        if (q->state == State::Done) return ZQD_OK; // too late: the result stands
        q->cancel.store(true);
        if (q->state != State::Queued) return ZQD_OK; // leaves its group before the next launch
        S->queue.erase(std::find(S->queue.begin(), S->queue.end(), q));
        S->in_use += q->est; // finish() releases it
    }
    S->finish(q, ZQD_ERR_CANCELLED, "CANCELLED", nullptr);
    return ZQD_OK;
}

static int wait_impl(zqd_server* S, uint64_t ticket, int64_t timeout_ms, zqd_result** out, double* latency_ms) {
    if (!S || !out) return zqd::fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    *out = nullptr;
    Req q;
    {
        std::unique_lock<std::mutex> lk(S->mu);
        auto it = S->live.find(ticket);
        if (it == S->live.end()) return zqd::fail(ZQD_ERR_NOT_FOUND, "UNKNOWN TICKET");
        q = it->second;
        auto ready = [&] { return q->state == State::Done; };
        if (timeout_ms < 0) S->cv_done.wait(lk, ready);
        else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
            return zqd::fail(ZQD_ERR_TIMEOUT, "REQUEST NOT DONE WITHIN THE TIMEOUT");
        S->live.erase(ticket);
    }
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(q->t1 - q->t0).count();
    if (q->status) return zqd::fail(q->status, q->error);
    *out = q->result;
    q->result = nullptr;
    return ZQD_OK;
}

extern "C" int zqd_server_wait(zqd_server* S, uint64_t ticket, zqd_result** out, double* latency_ms) {
    return wait_impl(S, ticket, -1, out, latency_ms);
}

extern "C" int zqd_server_wait_timeout(zqd_server* S, uint64_t ticket, uint32_t timeout_ms, zqd_result** out,
                                       double* latency_ms) {
    return wait_impl(S, ticket, (int64_t)timeout_ms, out, latency_ms);
}

extern "C" int zqd_server_poll(zqd_server* S, zqd_event* events, uint32_t max_events, uint32_t* count) {
    if (!S || !count || (!events && max_events)) return zqd::fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    std::lock_guard<std::mutex> lk(S->mu);
    S->polled.clear();
    const uint32_t n = (uint32_t)std::min<size_t>(max_events, S->events.size());
    for (uint32_t i = 0; i < n; ++i) {
        S->polled.push_back(std::move(S->events.front()));
        S->events.pop_front();
    }
    for (uint32_t i = 0; i < n; ++i) {
        const Event& e = S->polled[i];
        zqd_event& o = events[i];
        o.ticket = e.ticket;
        o.kind = e.kind;
        o.status = e.status;
        o.solve = e.solve;
        o.first_row = e.first_row;
        o.nrows = e.nrows;
        o.width = e.width;
        o.solve_finished = e.solve_finished;
        o.rows = e.rows.empty() ? nullptr : e.rows.data();
    }
    *count = n;
    return ZQD_OK;
}

extern "C" int zqd_server_stats_get(zqd_server* S, zqd_server_stats* out) {
    if (!S || !out) return zqd::fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->stats;
    out->device_bytes_in_use = S->in_use;
    out->queued = S->queue.size();
    out->pending_events = S->events.size();
    return ZQD_OK;
}

extern "C" void zqd_server_destroy(zqd_server* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    for (std::thread& t : S->workers) t.join();
    delete S;
}
