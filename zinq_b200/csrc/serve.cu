// serve.cu -- a job server for streams of independent propagation requests.
//
// Requests are validated and copied at submission.  Worker threads (one CUDA stream per job)
// admit them in arrival order while their estimated device memory fits the budget; waiting 1-D
// single-solve requests that share the head's kernel shape (precision, states, grid points) are
// taken with it and run as one grouped launch of the resident line kernel (continuous batching),
// the rest run on their own.  N-D jobs launch directly (a one-shot job gains nothing from graph
// capture).  Results and the submit-to-completion latency are handed back by zqd_server_wait.
// The reference has no serving layer: this is the request loop around its quantum_dynamics.run.
#include <algorithm>
#include <chrono>
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

struct Request {
    uint64_t ticket = 0;
    zqd::Opts o;
    size_t est = 0;          // estimated device bytes while it runs
    uint64_t group_key = 0;  // 0: runs alone; else requests with equal keys share a launch
    Clock::time_point t0, t1;
    int status = ZQD_OK;
    std::string error;
    zqd_result* result = nullptr;
    bool done = false;
    ~Request() {
        if (result) zqd_result_destroy(result);
    }
};

// Upper bound of a job's device allocations (tables, wavefunction copies, history, scratch).
size_t estimate_bytes(const zqd::Opts& o) {
    size_t N = 1;
    for (uint32_t i = 0; i < o.ndim; ++i) N *= o.npoint;
    const size_t S = (size_t)o.pot_ns, c = o.precision == ZQD_FP32_MIXED ? 8 : 16, nsolve = o.imag_nstate ? o.imag_nstate : 1;
    const size_t nsym = S * (S + 1) / 2;
    size_t b = (4 + nsolve) * S * N * c;                  // psi, phi, psi0, initial state, relaxed states
    b += nsym * N * 16 + N * 16 + 2 * S * S * N * 8 + N * 8; // R, kinetic phase, V and U, cap weights
    b += nsolve * ((size_t)o.iterations + 1) * (size_t)zqd::RowLayout{(int)o.ndim, (int)S}.width() * 8;
    b += N / 4 * 8 * 48 + (1u << 20);                     // partial sums, small tables, slack
    return b;
}

uint64_t group_key(const zqd::Opts& o) {
    if (o.ndim != 1 || o.imag_nstate > 1) return 0;
    return 1 + ((uint64_t)o.npoint << 8) + ((uint64_t)o.pot_ns << 2) + (o.precision == ZQD_FP32_MIXED ? 2 : 0);
}

} // namespace

struct zqd_server {
    int device = 0;
    size_t budget = 0, in_use = 0, peak = 0;
    uint32_t max_batch = 16;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
    uint64_t next_ticket = 1;
    bool stop = false;
    zqd_server_stats stats{};
    std::vector<std::thread> workers;

    void work();
    void run(std::vector<std::shared_ptr<Request>>& batch);
};

void zqd_server::run(std::vector<std::shared_ptr<Request>>& batch) {
    std::vector<zqd_job*> jobs(batch.size(), nullptr);
    std::vector<int> rc(batch.size(), ZQD_OK);
    std::vector<std::string> err(batch.size());
    for (size_t i = 0; i < batch.size(); ++i) {
        zqd::Opts o = batch[i]->o;
        rc[i] = zqd::job_create_opts(std::move(o), &jobs[i]);
        if (rc[i]) err[i] = zqd::last_error();
        else jobs[i]->nd_use_graph = false;
    }
    // one grouped launch per precision (ZQD_PRECISION_AUTO requests resolve at creation)
    std::vector<zqd_job*> group[2];
    for (size_t i = 0; i < batch.size(); ++i)
        if (!rc[i] && batch[i]->group_key) group[jobs[i]->fp32 ? 1 : 0].push_back(jobs[i]);
    int grc[2] = {ZQD_OK, ZQD_OK};
    std::string gerr[2];
    for (int g = 0; g < 2; ++g)
        if (group[g].size() > 1) {
            grc[g] = zqd::run_line_group(group[g], group[g][0]->stream, nullptr);
            if (grc[g]) gerr[g] = zqd::last_error();
        }
    for (size_t i = 0; i < batch.size(); ++i) {
        if (rc[i]) continue;
        const int g = jobs[i]->fp32 ? 1 : 0;
        const bool grouped = group[g].size() > 1 && batch[i]->group_key;
        if (grouped) {
            rc[i] = grc[g];
            err[i] = gerr[g];
        } else if ((rc[i] = zqd_job_run(jobs[i]))) {
            err[i] = zqd::last_error();
        }
        if (!rc[i] && (rc[i] = zqd_job_result(jobs[i], &batch[i]->result))) err[i] = zqd::last_error();
    }
    for (zqd_job* J : jobs) zqd_job_destroy(J);
    std::lock_guard<std::mutex> lk(mu);
    const Clock::time_point t1 = Clock::now();
    for (size_t i = 0; i < batch.size(); ++i) {
        Request& q = *batch[i];
        q.status = rc[i];
        q.error = err[i];
        q.t1 = t1;
        q.done = true;
        in_use -= q.est;
        ++stats.completed;
        if (rc[i]) ++stats.failed;
    }
    for (int g = 0; g < 2; ++g)
        if (group[g].size() > 1) {
            ++stats.grouped_launches;
            stats.grouped_jobs += group[g].size();
        }
    cv_done.notify_all();
    cv_work.notify_all();
}

void zqd_server::work() {
    cudaSetDevice(device);
    for (;;) {
        std::vector<std::shared_ptr<Request>> batch;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return (stop && queue.empty()) || (!queue.empty() && in_use + queue.front()->est <= budget); });
            if (queue.empty()) return;
            // the head, then waiting requests of its group while they fit (arrival order)
            std::shared_ptr<Request> head = queue.front();
            queue.pop_front();
            batch.push_back(head);
            in_use += head->est;
            if (head->group_key)
                for (auto it = queue.begin(); it != queue.end() && batch.size() < max_batch;) {
                    if ((*it)->group_key == head->group_key && in_use + (*it)->est <= budget) {
                        in_use += (*it)->est;
                        batch.push_back(*it);
                        it = queue.erase(it);
                    } else {
                        ++it;
                    }
                }
            peak = std::max(peak, in_use);
            stats.peak_device_bytes = peak;
            if (!queue.empty()) cv_work.notify_one();
        }
        run(batch);
    }
}

extern "C" void zqd_server_config_init(zqd_server_config* cfg) {
    if (!cfg) return;
    *cfg = zqd_server_config{};
    cfg->struct_size = sizeof(zqd_server_config);
    cfg->workers = 4;
    cfg->max_batch = 16;
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
    size_t free_b = 0, total_b = 0;
    ZQD_CUDA(cudaMemGetInfo(&free_b, &total_b));
    S->budget = cfg->device_budget_bytes ? (size_t)cfg->device_budget_bytes : free_b / 10 * 9;
    S->max_batch = std::max(1u, cfg->max_batch ? cfg->max_batch : 16u);
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

extern "C" int zqd_server_wait(zqd_server* S, uint64_t ticket, zqd_result** out, double* latency_ms) {
    if (!S || !out) return zqd::fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    *out = nullptr;
    std::shared_ptr<Request> q;
    {
        std::unique_lock<std::mutex> lk(S->mu);
        auto it = S->live.find(ticket);
        if (it == S->live.end()) return zqd::fail(ZQD_ERR_NOT_FOUND, "UNKNOWN TICKET");
        q = it->second;
        S->cv_done.wait(lk, [&] { return q->done; });
        S->live.erase(it);
    }
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(q->t1 - q->t0).count();
    if (q->status) return zqd::fail(q->status, q->error);
    *out = q->result;
    q->result = nullptr;
    return ZQD_OK;
}

extern "C" int zqd_server_stats_get(zqd_server* S, zqd_server_stats* out) {
    if (!S || !out) return zqd::fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->stats;
    out->device_bytes_in_use = S->in_use;
    out->queued = S->queue.size();
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
