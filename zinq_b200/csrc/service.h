// service.h -- host side of the persistent line-service kernel (line_service_kernel).
//
// One LineServiceHost per (precision, state count): a table of job descriptors, end flags and row
// counters in pinned host memory that the device reads and writes directly, a claim counter in
// device memory, and the launches of the persistent kernel working through the table.  post()
// appends a created single-CTA 1-D job; the kernels claim jobs in posting order, each running a
// whole solve, and publish every history row and the end of each solve; poll() reports them.  A
// kernel whose CTAs found no work for idle_us exits; pump() launches again whenever posted jobs
// wait unclaimed and fewer than max_ctas CTAs are alive.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "job.h"

namespace zqd {

class LineServiceHost {
  public:
    // kernels of `threads` threads and `smem` bytes of dynamic shared memory per CTA: jobs whose
    // single-CTA shape needs at most that (small lines share an SM, the largest take one each)
    LineServiceHost(bool fp32, int S, int threads, size_t smem) : fp32_(fp32), S_(S), threads_(threads), smem_(smem) {}
    ~LineServiceHost();
    int init(unsigned capacity, unsigned max_ctas, double idle_us);
    // slots free for post() (a slot is free again after release())
    unsigned free_slots() const { return capacity_ - (unsigned)(posted_ - released_); }
    // appends job J (created with a single-CTA shape); *slot receives its table slot
    int post(zqd_job* J, unsigned* slot);
    // rows published so far for the job in `slot`, and whether its solve has ended
    int rows(unsigned slot) const;
    bool ended(unsigned slot) const;
    // the job in `slot` has been handed back: its slot may be reused (in posting order)
    void release(unsigned slot);
    // launch kernels while posted jobs wait unclaimed; reap the launches that ended
    int pump();
    // every kernel of this service has ended (after close())
    bool idle();
    void close(); // kernels exit once every posted job is claimed
    unsigned idle_exits() const;
    unsigned launches() const { return launches_; }
    int launch(unsigned grid); // one more kernel of `grid` CTAs on the table

  private:
    struct Launch {
        cudaEvent_t end = nullptr;
        unsigned grid = 0;
    };
    bool fp32_;
    int S_, threads_;
    size_t smem_;
    unsigned capacity_ = 0, max_ctas_ = 0, launches_ = 0;
    unsigned long long posted_ = 0, released_ = 0;
    long long idle_cycles_ = 0;
    size_t desc_bytes_ = 0;
    char* descs_ = nullptr;            // pinned, [capacity][desc_bytes]
    unsigned* ctl_ = nullptr;          // pinned LineServiceCtl words
    int* done_ = nullptr;              // pinned [capacity]
    int* progress_ = nullptr;          // pinned [capacity]
    unsigned* claim_ = nullptr;        // device
    std::vector<char> freed_;          // slots released out of order
    std::vector<Launch> live_;
    cudaStream_t st_ = nullptr;
    unsigned claimed(); // jobs claimed so far (read after the launches that claim have ended)
};

} // namespace zqd
