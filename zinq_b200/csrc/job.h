// job.h -- the job handle behind the C-ABI, shared by the 1-D and N-D drivers.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "internal.h"

namespace zqd {

// device allocation owned by a job
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool owned = true;         // false: a view into another buffer (not freed here)
    cudaStream_t st = nullptr; // allocated (and freed) in this stream; null: complete on return
    ~DevBuf() { release(); }
    void release() {
        if (owned) dev_free(p, st);
        p = nullptr;
        bytes = 0;
    }
    // a view of b bytes at base (null when b is 0), owned by another DevBuf
    void view(void* base, size_t b) {
        release();
        p = b ? base : nullptr;
        bytes = b;
        owned = false;
    }
    int alloc(size_t b, cudaStream_t stream = nullptr) {
        release();
        owned = true;
        st = stream;
        bytes = b;
        if (b == 0) return ZQD_OK;
        cudaError_t e = dev_alloc(&p, b, stream);
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(ZQD_ERR_DEVICE_OOM, std::string("cudaMalloc(") + std::to_string(b) + "): " + cudaGetErrorString(e));
        }
        return ZQD_OK;
    }
    template <typename X> X* as() const { return reinterpret_cast<X*>(p); }
};

} // namespace zqd

struct zqd_job;
namespace zqd {
// stream: the job's work and buffers go to this stream, which the caller owns and keeps until
// the job is destroyed (null: the job creates its own)
int job_create_opts(Opts&& o, zqd_job** out, cudaStream_t stream = nullptr);
int run_line_group(const std::vector<zqd_job*>& jobs, cudaStream_t st, float* ms);
int step_line_group(const std::vector<zqd_job*>& jobs, uint32_t nsteps, cudaStream_t st);
// the persistent service kernel's side of a job (service.cu)
size_t line_desc_bytes(bool fp32);
int service_desc(zqd_job* J, void* out, int* progress);
int service_job_ended(zqd_job* J);
void service_job_rows(zqd_job* J, int rows);

// Launch shape chosen by the autotuner (tune.cu) for a (dims, points, states, precision) key, or
// forced on this thread while the autotuner measures a candidate; zero fields keep the default.
struct ShapeOverride {
    int C = 0, lrmax = 0; // 1-D: CTAs per cluster, log2 of the largest local radix
    int rows = 0, tile = 0; // N-D: rows of the last axis per row-pass CTA, lines per tile-pass CTA
    int tma_w = 0;          // N-D: lines per TMA-staged tile (-1: the earlier tile kernel)
    int tma_rows = 0;       // N-D: rows per TMA-staged row block (-1: the earlier row kernel)
};
bool lookup_shape(int d, int n, int S, bool fp32, ShapeOverride& out);
// a job created with a given launch shape (the autotuner's candidates, the service's single CTAs)
int job_create_shaped(Opts&& o, const ShapeOverride& shape, zqd_job** out, cudaStream_t stream = nullptr);
// Time-dependent potential whose eigenvector signs some output observes: the wavefunction history in
// the adiabatic basis, or the toDia of a later imaginary-time solve (wavepacket.zig:145-167 then apply).
inline bool needs_sign_tracking(const Opts& o, int S, int nsolve) {
    return o.pot_td && S > 1 &&
           (((o.write_mask & ZQD_WRITE_WAVEFUNCTION) && o.adiabatic) || (o.ic_adiabatic && nsolve > 1));
}
} // namespace zqd

struct zqd_job {
    zqd::Opts o;
    int S = 1, d = 1, n = 0;
    size_t N = 0;
    int C = 1, m = 0, q = 0, E = 8, threads = 32;
    size_t smem = 0;
    bool fp32 = false;
    bool r_global = false; // 1-D: R read from global memory (the largest lines)
    int lrmax = 3;         // 1-D: log2 of the largest local radix
    bool u_smem = false;   // 1-D: the shape stages the eigenvectors in shared memory
    int nsolve = 1, hc = 0;
    zqd::PotStore pot;
    cudaStream_t stream = nullptr;
    bool own_stream = true; // false: the caller's stream (the server's per-worker streams)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    zqd::DevBuf R, expk, V, U, capw, tw, psi_save, psi0, orth, hist, fin, rows, jobs, scratch;
    zqd::DevBuf phi, part, book, flags; // N-D grids: momentum scratch, partial sums, bookkeeping, stop flags
    zqd::DevBuf psi_init;               // initial wavefunction replacing the Gaussian (1-D: permuted layout)
    zqd::DevBuf wfn_hist;               // write.wavefunction: [solve][step][S][N] (1-D: permuted layout)
    zqd::DevBuf sgn;                    // eigenvector overlaps with the previous update (sign tracking)
    zqd::DevBuf carry, done;            // 1-D: absorbed populations between launches; per-solve end flags
    zqd::DevBuf arena;                  // 1-D jobs: one pool block holding the buffers above (views)
    double min_gap = -1;                // ZQD_PRECISION_AUTO: smallest adiabatic gap on the grid (-1: not computed)
    int nd_rows = 1, nd_tile = 8, nd_row_threads = 32, nd_tile_threads = 32, nd_row_bufs = 2;
    // N-D strided-axis passes through the TMA-staged persistent kernel: lines per tile (log2), CTAs,
    // and one tensor map (CUtensorMap, 128 bytes) over psi per strided axis
    bool nd_tma = false;
    int nd_tma_logW = 0, nd_tma_ctas = 0;
    int nd_tma_ctas_full = 0; // the momentum-sum launches' grid: every resident CTA (never capped)
    alignas(64) unsigned char nd_maps[2][128] = {};
    alignas(64) unsigned char nd_maps_phi[2][128] = {}; // the same over phi (the momentum passes)
    // the row pass's TMA-staged persistent form: rows per block (log2), CTAs, tensor map over psi
    bool nd_row_tma = false;
    bool nd_row_tma_phi = false; // the momentum-copy launches too (else they take the earlier kernel)
    int nd_row_tma_logL = 0, nd_row_tma_ctas = 0;
    alignas(64) unsigned char nd_row_map[128] = {};
    alignas(64) unsigned char nd_row_map_phi[128] = {}; // the same over phi (the momentum copy)
    cudaGraphExec_t nd_graph = nullptr; // the whole N-D run, captured on its first call and replayed after
    bool nd_use_graph = true;           // false: launch directly (one-shot jobs skip the capture cost)
    float last_ms = 0;
    int runs = 0; // runs started (a time-dependent potential's tables are rebuilt for every later run)
    // step-wise progress (zqd_job_step): the solve in progress, rows recorded per solve, solves ended
    int step_solve = 0;
    std::vector<int> solve_rows; // rows of each solve's history written so far
    std::vector<char> solve_ended;
    bool stepping = false; // a step-wise run is in progress
    bool fetch_psi = true; // zqd_job_result downloads the final wavefunctions
    // zqd_job_observables cursor and its host buffer
    int obs_solve = 0, obs_row = 0;
    std::vector<double> obs_buf;
    size_t device_bytes = 0;
    uint64_t h2d = 0, d2h = 0; // bytes copied by this job
    // The buffers go back to the pool in the job's stream order, without waiting: the job's work in
    // other streams (group launches, the service kernel) has been waited for by whoever launched it.
    ~zqd_job() {
        zqd::DevBuf* bufs[] = {&R,   &expk, &V,    &U,        &capw,     &tw,  &psi_save, &psi0,  &orth,
                               &hist, &fin, &rows, &jobs,     &scratch,  &phi, &part,     &book,  &flags,
                               &psi_init, &wfn_hist, &sgn, &carry, &done, &arena};
        for (zqd::DevBuf* b : bufs) b->release();
        pot.release();
        if (nd_graph) cudaGraphExecDestroy(nd_graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream && own_stream) cudaStreamDestroy(stream);
    }
};
