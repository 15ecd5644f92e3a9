// internal.h -- host-side state shared by the C-ABI implementation files.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/zinq_qd.h"
#include "expr.h"
#include "physics.cuh"

namespace zqd {

void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
const char* last_error();

// Device buffers of jobs come from the device's stream-ordered memory pool: cudaFree waits for
// every stream of the device, which would stall concurrent jobs (the server runs several at a
// time); a pool free waits for nothing.  Freed blocks stay cached in the pool for later jobs.
// With a stream, allocation and free are ordered in that stream (the buffer is usable by work
// queued there after the call, and by other streams once it has been synchronised); without
// one, the allocation is complete when the call returns.  A stream that shares a hardware
// queue with busy streams would make a synchronising call wait for their work too, so jobs
// allocate in their own stream.
cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t st = nullptr);
void dev_free(void* p, cudaStream_t st = nullptr);
// The mbarrier wait budget (SM cycles) of the next launch of an N-D TMA-staged pass, and whether
// that launch withholds each CTA's first load (zqd_testing_tma_withhold_load); the default budget
// and false unless a test armed it.
long long tma_wait_budget(long long default_cycles, bool* withhold);
// device memory this process can still allocate: free HBM plus the blocks the pool keeps for reuse
size_t device_free_bytes();

#define ZQD_CUDA(call)                                                                                             \
    do {                                                                                                           \
        cudaError_t e__ = (call);                                                                                  \
        if (e__ != cudaSuccess)                                                                                    \
            return ::zqd::fail(e__ == cudaErrorMemoryAllocation ? ZQD_ERR_DEVICE_OOM : ZQD_ERR_DEVICE,             \
                               std::string(#call) + ": " + cudaGetErrorString(e__));                               \
    } while (0)

// Deep copy of zqd_options (the caller's memory is only borrowed during a call).
struct Opts {
    uint32_t ndim = 0, npoint = 0;
    std::vector<double> bounds, pos, mom, gamma, mass, cap_bounds;
    uint32_t ic_state = 0;
    bool ic_adiabatic = false;
    double time_step = 0;
    uint32_t iterations = 0, write_mask = 0, log_interval = 1, imag_nstate = 0, spectrum_padding = 0;
    bool adiabatic = false, has_cap = false, cap_track = false, cap_has_stop = false, has_spectrum = false, log = false;
    double cap_exponent = 0.001, cap_stop_norm = 0, spectrum_threshold = 1e-6;
    zqd_precision precision = ZQD_FP64;
    std::vector<double> ic_wfn; // 2 * S * N doubles when an initial wavefunction is given
    // potential
    int pkind = 0;
    std::vector<double> harmonic_k;
    double p[5] = {0, 0, 0, 0, 0};
    std::vector<std::string> custom;
    uint32_t custom_ns = 0, custom_nd = 0;
    bool custom_td = false;
    std::vector<double> lvc_freq, lvc_exc, lvc_kappa, lvc_lambda;
    std::vector<double> file_table;
    uint32_t file_nrow = 0, file_ncol = 0, file_nd = 0;
    // derived
    int pot_nd = 0, pot_ns = 0;
    bool pot_td = false;
    // set by the job server: resident CTAs per SM that an N-D job's persistent (TMA-staged) tile
    // pass uses, so that the jobs it runs side by side can interleave (0: as many as fit)
    int tma_ctas_per_sm = 0;
};

int copy_options(const zqd_options* in, Opts& o);
int validate(const Opts& o);

// Device resident potential description + its storage.
struct PotStore {
    PotDev dev{};
    void* d_blob = nullptr; // the potential's device data (program, constants or tables) in one block
    size_t bytes = 0;       // uploaded to the device
    cudaStream_t st = nullptr; // the stream the block was allocated (and is freed) in
    void release();
    ~PotStore() { release(); }
};
// st: the stream of the job that uses the potential (null: complete on return)
int build_potential(const Opts& o, PotStore& ps, cudaStream_t st = nullptr);

// Twiddle tables exp(-2 pi i t / n), t < n, generated in long double and rounded.
std::vector<double> twiddles_f64(int n);

struct SolveOut {
    size_t rows = 0;
    std::vector<double> hist; // rows x HC
    std::vector<double> fin;  // HC
    std::vector<double> psi;  // S x N complex, natural order
    std::vector<double> acfpad, sigma;
    std::vector<double> wfn; // write.wavefunction: rows x S x N complex, natural order
};

// calcSpectrum of one solve from its device history (spectrum.cu)
int spectrum_device(cudaStream_t st, const double* d_hist, int hc, int col, size_t rows, const Opts& o, SolveOut& so,
                    uint64_t& d2h);

} // namespace zqd

struct zqd_result {
    uint32_t ndim = 0, nstate = 0;
    uint64_t npoint_total = 0;
    std::vector<zqd::SolveOut> solves;
    std::vector<std::vector<double>> series_cache; // per (solve, series)
    double device_ms = 0;
    zqd_precision precision = ZQD_FP64; // the form the job ran in
    uint32_t write_mask = 0;
    double time_step = 0;
    std::vector<double> grid; // bounds [ndim][2] and npoint, for the wavefunction file's coordinates
    int hc = 0;
    uint64_t h2d = 0, d2h = 0;
};
