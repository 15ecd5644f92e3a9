// serve.cu -- a job server for streams of independent propagation requests.
//
// Requests are validated and copied at submission.  Worker threads (one CUDA stream each, which
// their jobs use for all their work and buffers) admit them in arrival order while their estimated device memory fits the budget and the
// device's measured free memory.  A worker advances its jobs in launches of `stream_steps`
// steps (zqd_job_step): 1-D single-solve requests that share a kernel shape (precision, states,
// grid points) form one group advanced by one launch of the resident line kernel, every member
// from its own step; between launches finished or cancelled members leave and waiting requests
// of the same shape join (continuous batching).  Other requests run on their own.  After every
// launch the new observable rows of each job are posted as events (zqd_server_poll); completion,
// failure and cancellation are events too, and zqd_server_wait hands the result over.
// 1-D single-solve requests whose line fits one CTA go to the persistent line-service kernel
// instead (service.h): resident CTAs claim them from a table in pinned memory as they are posted
// and publish every row; a poller thread streams those rows and completes the requests.
// The reference has no serving layer: this is the request loop around its quantum_dynamics.run.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <map>
#include <thread>
#include <tuple>
#include <unordered_map>

#include "internal.h"
#include "job.h"
#include "line_kernel.cuh"
#include "service.h"

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

// The first non-finite entry of the recorded columns (the others are NaN by design) of new rows,
// described for the error message; empty when every entry is finite.
std::string nonfinite_entry(const zqd_obs_rows& r, int d, int S, uint32_t wmask) {
    const zqd::RowLayout L{d, S};
    for (uint32_t k = 0; k < r.nrows; ++k) {
        const double* row = r.rows + (size_t)k * r.width;
        int col = -1;
        if ((wmask & ZQD_WRITE_NORM) && !std::isfinite(row[L.norm()])) col = L.norm();
        if (wmask & ZQD_WRITE_POPULATION)
            for (int s = 0; s < S && col < 0; ++s)
                if (!std::isfinite(row[L.pop() + s])) col = L.pop() + s;
        if (col >= 0)
            return "NON-FINITE OBSERVABLE (step " + std::to_string(r.first_row + k) + ", row column " +
                   std::to_string(col) + ": " + std::to_string(row[col]) + ")";
    }
    return std::string();
}

} // namespace

// a request running on the persistent line-service kernel
struct SvcJob {
    Req q;
    zqd::LineServiceHost* host = nullptr;
    unsigned slot = 0;
    int streamed = 0; // rows already posted as events
};

// service tables per (precision, states, threads per CTA, shared memory per CTA)
using SvcKey = std::tuple<int, int, int, size_t>;

struct zqd_server {
    int device = 0;
    size_t budget = 0, in_use = 0, peak = 0;
    uint32_t max_batch = 16, stream_steps = 256, max_events = 65536;
    bool stream_rows = true;
    bool fetch_psi = true; // results carry the final wavefunction
    // persistent line service: one table per (precision, states), guarded by svc_mu
    bool use_service = true;
    uint32_t service_ctas = 0;
    double service_idle_us = 200.0;
    std::mutex svc_mu;
    std::condition_variable svc_cv;
    std::map<SvcKey, std::unique_ptr<zqd::LineServiceHost>> svc;
    std::vector<SvcJob> svc_jobs;
    bool svc_stop = false;
    std::thread svc_thread;
    bool try_service(const Req& q); // true: the service took the request (or it failed there); false: keep it
    void service_loop();
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

    // Device memory measured free (cudaMemGetInfo and the pool's spare blocks) at free_at, when this
    // server's admitted estimates summed to in_use_at.  A measurement takes milliseconds while kernels
    // run, so admission works from it and the estimates admitted or released since.
    mutable size_t free_bytes = 0, in_use_at = 0;
    mutable Clock::time_point free_at{};
    size_t free_estimate() const { // under mu
        const long long f = (long long)free_bytes + (long long)in_use_at - (long long)in_use;
        return f > 0 ? (size_t)f : 0;
    }
    bool fits(const Request& q) const; // under mu
    void refresh_free();               // measures without mu
    // Streams live as long as the server: a stream per worker, and one for the service's requests
    // (creation, row and result copies).  CUDA maps streams onto a few hardware queues; a stream
    // made per job would soon share one with another worker's busy stream, and every wait on it
    // (an allocation, a copy) would wait for that worker's kernels as well.
    cudaStream_t svc_io = nullptr;
    void work();
    void run_active(std::vector<Req> group, cudaStream_t ws);
    void post(Event&& e);                           // under mu
    void finish(const Req& q, int status, const std::string& err, zqd_result* res); // takes mu
    int stream(const Req& q, std::string& err); // ZQD_ERR_NUMERIC (err says where) for a non-finite row
};

// A request fits when its estimate stays within the budget and, with an eighth to spare, within the
// free device memory.  The free memory is measured again here only when the running estimate says
// no (at most every 20 ms); the service thread refreshes it while requests wait (refresh_free).
bool zqd_server::fits(const Request& q) const {
    if (in_use + q.est > budget) return false;
    if (in_use == 0) return true; // nothing of ours to wait for: the allocation decides
    const size_t need = q.est + q.est / 8;
    if (need <= free_estimate()) return true;
    const Clock::time_point now = Clock::now();
    if (now - free_at < std::chrono::milliseconds(20)) return false;
    free_bytes = zqd::device_free_bytes();
    free_at = now;
    in_use_at = in_use;
    return need <= free_bytes;
}

// Measures the free device memory without holding mu (other processes' use shows up here).  The
// estimates admitted meanwhile count as taken and those released meanwhile as still held: in_use_at
// is the smaller of the sums before and after the measurement.
void zqd_server::refresh_free() {
    size_t before;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (queue.empty() || in_use == 0) return; // nobody waits for admission
        before = in_use;
    }
    const size_t f = zqd::device_free_bytes();
    std::lock_guard<std::mutex> lk(mu);
    free_bytes = f;
    in_use_at = std::min(before, in_use);
    free_at = Clock::now();
    cv_work.notify_all();
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

// the job's observable rows recorded since the last call, as events (none without stream_rows)
int zqd_server::stream(const Req& q, std::string& err) {
    if (!stream_rows) return ZQD_OK; // no row events: the final observables are checked at the end
    for (;;) {
        zqd_obs_rows r{};
        if (zqd_job_observables(q->job, &r) != ZQD_OK || r.nrows == 0) return ZQD_OK;
        err = nonfinite_entry(r, (int)q->o.ndim, q->o.pot_ns, q->o.write_mask);
        if (!err.empty()) return ZQD_ERR_NUMERIC;
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
void zqd_server::run_active(std::vector<Req> group, cudaStream_t st) {
    const uint64_t key = group.front()->group_key;
    auto create = [&](const Req& q) -> bool {
        zqd::Opts o = q->o;
        // several workers' jobs share the device: one resident CTA per SM for the persistent tile pass
        o.tma_ctas_per_sm = 1;
        const int rc = zqd::job_create_opts(std::move(o), &q->job, st);
        if (rc) {
            finish(q, rc, zqd::last_error(), nullptr);
            q->job = nullptr;
            return false;
        }
        q->job->nd_use_graph = false;
        q->job->fetch_psi = fetch_psi;
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
                rc = stream(q, q->error);
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
}

// Single-solve 1-D requests whose line fits one CTA: created with the single-CTA shape and posted
// to the service table of their (precision, states).  False: the request stays with the worker.
bool zqd_server::try_service(const Req& q) {
    const zqd::Opts& o = q->o;
    const bool fp32_req = o.precision != ZQD_FP64;
    if (!use_service || o.ndim != 1 || o.imag_nstate > 1 || o.npoint > (fp32_req ? 2048u : 1024u)) return false;
    zqd::ShapeOverride one;
    one.C = 1;
    one.lrmax = 2;
    zqd_job* J = nullptr;
    zqd::Opts copy = o;
    if (const int rc = zqd::job_create_shaped(std::move(copy), one, &J, svc_io)) {
        if (rc == ZQD_ERR_UNSUPPORTED) return false; // the line does not fit one CTA: the general path
        finish(q, rc, zqd::last_error(), nullptr);   // e.g. device memory refused: the request fails here
        return true;
    }
    if (J->C != 1 || J->lrmax != 2) {
        zqd_job_destroy(J);
        return false;
    }
    J->fetch_psi = fetch_psi;
    // the job's shape, rounded up: threads to a power of two (>= 64), shared memory to 16 KiB
    int threads = 64;
    while (threads < J->threads) threads <<= 1;
    const size_t smem = (J->smem + 16383) / 16384 * 16384;
    std::lock_guard<std::mutex> lk(svc_mu);
    auto& host = svc[SvcKey{J->fp32 ? 1 : 0, J->S, threads, smem}];
    if (!host) {
        host.reset(new zqd::LineServiceHost(J->fp32, J->S, threads, smem));
        if (host->init(1024, service_ctas, service_idle_us)) {
            host.reset();
            zqd_job_destroy(J);
            return false;
        }
    }
    unsigned slot = 0;
    if (host->free_slots() == 0 || host->post(J, &slot)) {
        zqd_job_destroy(J);
        return false;
    }
    q->job = J;
    svc_jobs.push_back(SvcJob{q, host.get(), slot, 0});
    svc_cv.notify_one();
    return true;
}

// Streams the rows the service kernels publish and completes their requests.  The table's state
// (post, release, launches) changes under svc_mu; the rows and end flags are read from pinned memory
// and the copies and result downloads run without the lock, so workers can post meanwhile.
void zqd_server::service_loop() {
    cudaSetDevice(device);
    const int batch_rows = stream_steps ? (int)stream_steps : INT32_MAX;
    Clock::time_point refreshed = Clock::now();
    for (;;) {
        if (Clock::now() - refreshed > std::chrono::milliseconds(250)) { // free device memory for admission
            refresh_free();
            refreshed = Clock::now();
        }
        std::vector<SvcJob> snap;
        {
            std::unique_lock<std::mutex> lk(svc_mu);
            if (svc_jobs.empty()) {
                if (svc_stop) return;
                svc_cv.wait_for(lk, std::chrono::milliseconds(5));
                continue;
            }
            snap = svc_jobs;
        }
        bool progressed = false;
        std::vector<std::pair<Req, int>> streamed;                                  // new streamed counts
        std::vector<std::tuple<SvcJob, int, std::string, zqd_result*>> ended_jobs; // to complete
        for (SvcJob& sj : snap) {
            const int rows = sj.host->rows(sj.slot);
            const bool ended = sj.host->ended(sj.slot);
            int rc = ZQD_OK;
            std::string err;
            if (ended) rc = zqd::service_job_ended(sj.q->job);
            else zqd::service_job_rows(sj.q->job, rows);
            if (!rc && (ended || rows - sj.streamed >= batch_rows)) { // rows in pieces of stream_steps
                progressed = true;
                rc = stream(sj.q, err);
                streamed.emplace_back(sj.q, rows);
            }
            if (!ended) continue; // runs on until its solve ends, even when cancelled
            zqd_result* res = nullptr;
            if (!rc && (rc = zqd_job_result(sj.q->job, &res))) err = zqd::last_error();
            if (!rc) {
                zqd_observables ob{};
                zqd_result_final(res, 0, &ob);
                if (!std::isfinite(ob.norm)) {
                    rc = ZQD_ERR_NUMERIC;
                    err = "NON-FINITE OBSERVABLE (the wavefunction norm is NaN or Inf)";
                }
            }
            if (!rc && sj.q->cancel.load()) rc = ZQD_ERR_CANCELLED, err = "CANCELLED";
            if (rc && res) {
                zqd_result_destroy(res);
                res = nullptr;
            }
            zqd_job_destroy(sj.q->job);
            sj.q->job = nullptr;
            ended_jobs.emplace_back(sj, rc, err, res);
        }
        {
            std::lock_guard<std::mutex> lk(svc_mu);
            for (auto& p : streamed)
                for (SvcJob& sj : svc_jobs)
                    if (sj.q == p.first) sj.streamed = p.second;
            for (auto& e : ended_jobs) {
                const SvcJob& sj = std::get<0>(e);
                sj.host->release(sj.slot);
                svc_jobs.erase(std::find_if(svc_jobs.begin(), svc_jobs.end(), [&](const SvcJob& x) { return x.q == sj.q; }));
            }
            for (auto& kv : svc) kv.second->pump(); // relaunch while posted jobs wait unclaimed
        }
        for (auto& e : ended_jobs) finish(std::get<0>(e).q, std::get<1>(e), std::get<2>(e), std::get<3>(e));
        if (!progressed && ended_jobs.empty()) std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
}

void zqd_server::work() {
    cudaSetDevice(device);
    cudaStream_t ws = nullptr; // null if it cannot be had: the jobs then make their own
    if (cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        ws = nullptr;
    }
    struct Drop {
        cudaStream_t s;
        ~Drop() {
            if (s) cudaStreamDestroy(s);
        }
    } drop{ws};
    for (;;) {
        std::vector<Req> batch;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return (stop && queue.empty()) || (!queue.empty() && fits(*queue.front())); });
            if (queue.empty()) return;
            // the head, then waiting requests of its shape while they fit (arrival order)
            Req head = queue.front();
            queue.pop_front();
            in_use += head->est;
            peak = std::max(peak, in_use);
            stats.peak_device_bytes = peak;
            head->state = State::Running;
            if (!queue.empty()) cv_work.notify_one();
            lk.unlock();
            if (try_service(head)) {
                std::lock_guard<std::mutex> lk2(mu);
                ++stats.service_jobs;
                continue;
            }
            lk.lock();
            batch.push_back(head);
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
        run_active(std::move(batch), ws);
    }
}

extern "C" void zqd_server_config_init(zqd_server_config* cfg) {
    if (!cfg) return;
    *cfg = zqd_server_config{};
    cfg->struct_size = sizeof(zqd_server_config);
    cfg->workers = 8;
    cfg->max_batch = 16;
    cfg->stream_steps = 256;
    cfg->stream_rows = 1;
    cfg->max_events = 65536;
    cfg->persistent_lines = 1;
    cfg->fetch_wavefunction = 1;
    cfg->service_ctas = 64;
    cfg->service_idle_us = 200.0;
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
    S->free_bytes = free_b;
    S->free_at = Clock::now();
    S->budget = cfg->device_budget_bytes ? (size_t)cfg->device_budget_bytes : free_b / 10 * 9;
    S->max_batch = std::max(1u, cfg->max_batch ? cfg->max_batch : 16u);
    S->stream_steps = cfg->stream_steps;
    S->stream_rows = cfg->stream_rows != 0;
    S->max_events = std::max(1u, cfg->max_events ? cfg->max_events : 65536u);
    S->stats.device_budget_bytes = S->budget;
    S->use_service = cfg->persistent_lines != 0;
    S->fetch_psi = cfg->fetch_wavefunction != 0;
    S->service_ctas = cfg->service_ctas;
    S->service_idle_us = cfg->service_idle_us > 0 ? cfg->service_idle_us : 200.0;
    if (cudaStreamCreateWithFlags(&S->svc_io, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        S->svc_io = nullptr; // the service's requests make their own streams
    }
    S->svc_thread = std::thread([s = S.get()] { s->service_loop(); });
    const uint32_t nw = std::max(1u, cfg->workers ? cfg->workers : 8u);
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
    uint64_t launches = 0;
    {
        std::lock_guard<std::mutex> lk(S->svc_mu);
        for (auto& kv : S->svc) launches += kv.second->launches();
    }
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->stats;
    out->device_bytes_in_use = S->in_use;
    out->queued = S->queue.size();
    out->pending_events = S->events.size();
    out->service_launches = launches;
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
    {
        std::lock_guard<std::mutex> lk(S->svc_mu);
        S->svc_stop = true;
    }
    S->svc_cv.notify_all();
    if (S->svc_thread.joinable()) S->svc_thread.join(); // every service request has completed
    S->svc.clear();
    if (S->svc_io) cudaStreamDestroy(S->svc_io);
    delete S;
}
