// service.cu -- host side of the persistent line-service kernel (see service.h).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <thread>

#include "internal.h"
#include "line_solve.cuh"
#include "service.h"

namespace zqd {

// launchers compiled in line_inst.cu, one translation unit per (precision, states)
int launch_service_d1(const void*, unsigned, int, size_t, cudaStream_t);
int launch_service_d2(const void*, unsigned, int, size_t, cudaStream_t);
int launch_service_d3(const void*, unsigned, int, size_t, cudaStream_t);
int launch_service_d4(const void*, unsigned, int, size_t, cudaStream_t);
int launch_service_f1(const void*, unsigned, int, size_t, cudaStream_t);
int launch_service_f2(const void*, unsigned, int, size_t, cudaStream_t);
int launch_service_f3(const void*, unsigned, int, size_t, cudaStream_t);
int launch_service_f4(const void*, unsigned, int, size_t, cudaStream_t);

LineServiceHost::~LineServiceHost() {
    close();
    for (Launch& l : live_) {
        cudaEventSynchronize(l.end); // bounded: the kernels exit once every posted job is claimed
        cudaEventDestroy(l.end);
    }
    if (st_) cudaStreamDestroy(st_);
    if (descs_) cudaFreeHost(descs_);
    if (ctl_) cudaFreeHost(ctl_);
    if (done_) cudaFreeHost(done_);
    if (progress_) cudaFreeHost(progress_);
    dev_free(claim_);
}

int LineServiceHost::init(unsigned capacity, unsigned max_ctas, double idle_us) {
    capacity_ = capacity;
    desc_bytes_ = line_desc_bytes(fp32_); // the kernel indexes the table as LineJob<T>[capacity]
    ZQD_CUDA(cudaHostAlloc((void**)&descs_, (size_t)capacity * desc_bytes_, cudaHostAllocMapped));
    ZQD_CUDA(cudaHostAlloc((void**)&ctl_, sizeof(LineServiceCtl), cudaHostAllocMapped));
    ZQD_CUDA(cudaHostAlloc((void**)&done_, capacity * sizeof(int), cudaHostAllocMapped));
    ZQD_CUDA(cudaHostAlloc((void**)&progress_, capacity * sizeof(int), cudaHostAllocMapped));
    std::memset(ctl_, 0, sizeof(LineServiceCtl));
    std::memset(done_, 0, capacity * sizeof(int));
    std::memset(progress_, 0, capacity * sizeof(int));
    freed_.assign(capacity, 0);
    ZQD_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    ZQD_CUDA(dev_alloc((void**)&claim_, 2 * sizeof(unsigned)));
    ZQD_CUDA(cudaMemsetAsync(claim_, 0, 2 * sizeof(unsigned), st_));
    ZQD_CUDA(cudaStreamSynchronize(st_));
    int dev = 0, sms = 148, khz = 1965000;
    ZQD_CUDA(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev);
    max_ctas_ = std::max(1u, std::min(max_ctas ? max_ctas : (unsigned)sms, (unsigned)sms));
    idle_cycles_ = (long long)(idle_us * 1e-3 * (double)khz); // clock64 counts SM cycles
    return ZQD_OK;
}

int LineServiceHost::post(zqd_job* J, unsigned* slot) {
    if (free_slots() == 0) return fail(ZQD_ERR_OUT_OF_MEMORY, "SERVICE TABLE FULL");
    const unsigned k = (unsigned)(posted_ % capacity_);
    int* prog_dev = nullptr;
    ZQD_CUDA(cudaHostGetDevicePointer((void**)&prog_dev, progress_ + k, 0));
    done_[k] = 0;
    progress_[k] = 0;
    if (int rc = service_desc(J, descs_ + (size_t)k * desc_bytes_, prog_dev)) return rc;
    // the descriptor and the cleared words are in memory before the device can see the new tail
    __atomic_store_n(&reinterpret_cast<LineServiceCtl*>(ctl_)->tail, (unsigned)(posted_ + 1), __ATOMIC_RELEASE);
    ++posted_;
    *slot = k;
    return pump();
}

int LineServiceHost::rows(unsigned slot) const { return __atomic_load_n(&progress_[slot], __ATOMIC_ACQUIRE); }
bool LineServiceHost::ended(unsigned slot) const { return __atomic_load_n(&done_[slot], __ATOMIC_ACQUIRE) != 0; }

void LineServiceHost::release(unsigned slot) {
    freed_[slot] = 1;
    while (released_ < posted_ && freed_[released_ % capacity_]) { // slots are reused in posting order
        freed_[released_ % capacity_] = 0;
        ++released_;
    }
}

int LineServiceHost::launch(unsigned grid) {
    LineService<double> svc{}; // the layout does not depend on T (pointers and scalars only)
    ZQD_CUDA(cudaHostGetDevicePointer((void**)&svc.jobs, descs_, 0));
    ZQD_CUDA(cudaHostGetDevicePointer((void**)&svc.ctl, ctl_, 0));
    ZQD_CUDA(cudaHostGetDevicePointer((void**)&svc.done, done_, 0));
    svc.counters = claim_;
    svc.capacity = capacity_;
    svc.idle_cycles = idle_cycles_;
    static_assert(sizeof(LineService<double>) == sizeof(LineService<float>), "service layouts differ");
    using Fn = int (*)(const void*, unsigned, int, size_t, cudaStream_t);
    static const Fn dt[4] = {launch_service_d1, launch_service_d2, launch_service_d3, launch_service_d4};
    static const Fn ft[4] = {launch_service_f1, launch_service_f2, launch_service_f3, launch_service_f4};
    if (int rc = (fp32_ ? ft : dt)[S_ - 1](&svc, grid, threads_, smem_, st_)) return rc;
    Launch l;
    l.grid = grid;
    ZQD_CUDA(cudaEventCreateWithFlags(&l.end, cudaEventDisableTiming));
    ZQD_CUDA(cudaEventRecord(l.end, st_));
    live_.push_back(l);
    ++launches_;
    return ZQD_OK;
}

// (with no service kernel alive, so the copy waits for nothing in the service's stream)
unsigned LineServiceHost::claimed() {
    unsigned c[2] = {0, 0};
    if (cudaMemcpyAsync(c, claim_, sizeof(c), cudaMemcpyDeviceToHost, st_) != cudaSuccess ||
        cudaStreamSynchronize(st_) != cudaSuccess)
        cudaGetLastError();
    return c[0];
}

int LineServiceHost::pump() {
    unsigned alive = 0;
    for (auto it = live_.begin(); it != live_.end();) {
        const cudaError_t q = cudaEventQuery(it->end);
        if (q == cudaErrorNotReady) {
            alive += it->grid;
            ++it;
            continue;
        }
        cudaEventDestroy(it->end);
        it = live_.erase(it);
        if (q != cudaSuccess) return fail(ZQD_ERR_DEVICE, std::string("service kernel: ") + cudaGetErrorString(q));
    }
    if (alive >= max_ctas_) return ZQD_OK;
    // jobs that no CTA has started (with kernels alive: an upper bound, from the rows published)
    unsigned long long waiting = 0;
    if (alive == 0) {
        waiting = posted_ - claimed();
    } else {
        for (unsigned long long j = released_; j < posted_; ++j) {
            const unsigned k = (unsigned)(j % capacity_);
            if (!freed_[k] && rows(k) == 0 && !ended(k)) ++waiting;
        }
        waiting = waiting > alive ? waiting - alive : 0;
    }
    if (waiting == 0) return ZQD_OK;
    return launch((unsigned)std::min<unsigned long long>(waiting, max_ctas_ - alive));
}

bool LineServiceHost::idle() {
    pump();
    return live_.empty();
}

void LineServiceHost::close() {
    if (ctl_) __atomic_store_n(&reinterpret_cast<LineServiceCtl*>(ctl_)->closed, 1u, __ATOMIC_RELEASE);
}

unsigned LineServiceHost::idle_exits() const {
    unsigned c[2] = {0, 0};
    if (cudaMemcpyAsync(c, claim_, sizeof(c), cudaMemcpyDeviceToHost, st_) != cudaSuccess ||
        cudaStreamSynchronize(st_) != cudaSuccess)
        cudaGetLastError();
    return c[1];
}

} // namespace zqd

// A service kernel that is never given work: its CTAs wait for a post at most idle_us and exit on
// their own.  Tests the bounded wait of the persistent kernel (a producer that never posts).
extern "C" int zqd_testing_service_idle(zqd_precision precision, uint32_t nstate, uint32_t ctas, double idle_us,
                                        uint32_t* idle_exits, double* wall_ms) {
    if (nstate < 1 || nstate > 4 || (precision != ZQD_FP64 && precision != ZQD_FP32_MIXED) || ctas == 0 || !idle_exits)
        return zqd::fail(ZQD_ERR_INVALID_INPUT, "BAD ARGUMENT");
    zqd::LineServiceHost svc(precision == ZQD_FP32_MIXED, (int)nstate, 128, 48 * 1024);
    if (int rc = svc.init(16, ctas, idle_us)) return rc;
    const auto t0 = std::chrono::steady_clock::now();
    if (int rc = svc.launch(ctas)) return rc; // nothing is posted
    while (!svc.idle()) {
        if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(20))
            return zqd::fail(ZQD_ERR_TIMEOUT, "SERVICE KERNEL DID NOT EXIT");
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    if (wall_ms) *wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    *idle_exits = svc.idle_exits();
    return ZQD_OK;
}
