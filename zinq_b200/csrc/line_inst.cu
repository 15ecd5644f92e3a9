// line_inst.cu -- instantiations of the resident line kernel for one
// (precision, state count) pair.  The build compiles this file once per pair
// with -DZQD_T=<double|float> -DZQD_S=<1..4> -DZQD_LAUNCH=<symbol> -DZQD_SERVICE=<symbol>, so the
// heavy template instantiations spread over parallel nvcc processes.
#include <mutex>

#include "internal.h"
#include "line_solve.cuh"

#if !defined(ZQD_T) || !defined(ZQD_S) || !defined(ZQD_LAUNCH) || !defined(ZQD_SERVICE)
#error "line_inst.cu needs -DZQD_T, -DZQD_S, -DZQD_LAUNCH and -DZQD_SERVICE"
#endif

namespace zqd {

template <int C, int LRM, int MAXT = LineMaxThreads<ZQD_T>::value>
static int launch_one(const LaunchShape* J, const void* d_jobs, int njobs) {
    auto kern = line_solve_kernel<ZQD_T, ZQD_S, C, LRM, MAXT>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [&] {
        attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 215 * 1024);
        if (attr_err == cudaSuccess && C > 8)
            attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    ZQD_CUDA(attr_err);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C * njobs, 1, 1);
    cfg.blockDim = dim3(J->threads, 1, 1);
    cfg.dynamicSmemBytes = J->smem;
    cfg.stream = J->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ZQD_CUDA(cudaLaunchKernelEx(&cfg, kern, reinterpret_cast<const LineJob<ZQD_T>*>(d_jobs)));
    return ZQD_OK;
}

// A radix-4 launch of C-CTA clusters: FP32 CTAs of at most 256 threads take the form compiled for
// 256 threads (up to 255 registers, no spills; the FP32 kernel is otherwise compiled for 512-thread
// CTAs and 128 registers)
template <int C> static int launch_r4(const LaunchShape* J, const void* dj, int nj) {
    if (LineMaxThreads<ZQD_T>::value > 256 && J->threads <= 256) return launch_one<C, 2, 256>(J, dj, nj);
    return launch_one<C, 2>(J, dj, nj);
}

// Radix-4 kernels for every cluster size; radix 8 only with 16 CTAs, the one shape whose CTAs can
// hold more points than radix-4 threads allow (the longest lines)
int ZQD_LAUNCH(const LaunchShape* J, const void* dj, int nj) {
    if (J->lrmax == 3) {
        if (J->C == 16) return launch_one<16, 3>(J, dj, nj);
        return fail(ZQD_ERR_UNSUPPORTED, "RADIX-8 LINE PASSES ARE BUILT FOR CLUSTERS OF 16 ONLY");
    }
    switch (J->C) {
    case 1: return launch_r4<1>(J, dj, nj);
    case 2: return launch_r4<2>(J, dj, nj);
    case 4: return launch_r4<4>(J, dj, nj);
    case 8: return launch_r4<8>(J, dj, nj);
    case 16: return launch_r4<16>(J, dj, nj);
    default: return fail(ZQD_ERR_UNSUPPORTED, "CLUSTER SIZE MUST BE 1, 2, 4, 8 OR 16");
    }
}

// The persistent service kernel (single-CTA jobs, radix-4 local passes): grid CTAs of `threads`
// threads with `smem` bytes of dynamic shared memory each, on stream st.
// (always the form compiled for LineMaxThreads: its many small CTAs share SMs, which fewer
// registers per thread allow)
int ZQD_SERVICE(const void* svc, unsigned grid, int threads, size_t smem, cudaStream_t st) {
    auto kern = line_service_kernel<ZQD_T, ZQD_S, 2>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [&] { attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 215 * 1024); });
    ZQD_CUDA(attr_err);
    kern<<<grid, threads, smem, st>>>(*reinterpret_cast<const LineService<ZQD_T>*>(svc));
    ZQD_CUDA(cudaGetLastError());
    return ZQD_OK;
}

} // namespace zqd
