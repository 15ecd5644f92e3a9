// measure.cu -- on-chip denominators for the resident 1-D kernel's roofline.
//
// The resident line kernel keeps the wavefunction in shared memory for a whole solve, so DRAM does
// not bound it; its step is a chain of shared-memory passes separated by CTA and cluster barriers.
// zqd_measure_onchip measures, on the current device: the shared-memory bandwidth of one SM
// (128-bit loads and stores without bank conflicts, every SM busy), the latency of __syncthreads in
// a 256-thread CTA and of a barrier across a 16-CTA cluster.  Each timing kernel runs a fixed number
// of iterations (no waits on other CTAs beyond the barriers themselves).
#include <cooperative_groups.h>

#include "internal.h"

namespace cg = cooperative_groups;

namespace {

constexpr int kSmemWords = 8192; // float4 words: 128 KiB per CTA

__global__ void __launch_bounds__(1024) smem_bw_kernel(int rounds, unsigned long long* cycles, float* sink) {
    extern __shared__ float4 buf[];
    for (int i = threadIdx.x; i < kSmemWords; i += blockDim.x) buf[i] = make_float4(i, 0, 0, 0);
    __syncthreads();
    const unsigned long long t0 = clock64();
    float4 acc = make_float4(0, 0, 0, 0);
    for (int r = 0; r < rounds; ++r) {
#pragma unroll 4
        for (int i = threadIdx.x; i < kSmemWords; i += blockDim.x) { // a warp reads 512 contiguous bytes
            const float4 v = buf[i];
            acc.x += v.x;
            acc.y += v.y;
            buf[i] = make_float4(v.y, v.x, acc.x, acc.y);
        }
    }
    __syncthreads();
    const unsigned long long t1 = clock64();
    if (threadIdx.x == 0) {
        cycles[blockIdx.x] = t1 - t0;
        sink[blockIdx.x] = acc.x + buf[0].z;
    }
}

__global__ void syncthreads_kernel(int rounds, unsigned long long* cycles, int* sink) {
    __shared__ int v;
    if (threadIdx.x == 0) v = 0;
    __syncthreads();
    const unsigned long long t0 = clock64();
    for (int r = 0; r < rounds; ++r) {
        if (threadIdx.x == (r & 255)) v += r;
        __syncthreads();
    }
    const unsigned long long t1 = clock64();
    if (threadIdx.x == 0) {
        cycles[blockIdx.x] = t1 - t0;
        sink[blockIdx.x] = v;
    }
}

__global__ void cluster_barrier_kernel(int rounds, unsigned long long* cycles) {
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    const unsigned long long t0 = clock64();
    for (int r = 0; r < rounds; ++r) cl.sync();
    const unsigned long long t1 = clock64();
    if (threadIdx.x == 0) cycles[blockIdx.x] = t1 - t0;
}

} // namespace

extern "C" int zqd_measure_onchip(zqd_onchip* out) {
    if (!out) return zqd::fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    int dev = 0, sms = 0, khz = 0;
    ZQD_CUDA(cudaGetDevice(&dev));
    ZQD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    ZQD_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev));
    unsigned long long* d_cyc = nullptr;
    float* d_sink = nullptr;
    ZQD_CUDA(cudaMalloc(&d_cyc, 4096 * sizeof(unsigned long long)));
    ZQD_CUDA(cudaMalloc(&d_sink, 4096 * sizeof(float)));
    std::vector<unsigned long long> cyc(4096);
    cudaEvent_t e0, e1;
    ZQD_CUDA(cudaEventCreate(&e0));
    ZQD_CUDA(cudaEventCreate(&e1));
    auto cleanup = [&] {
        cudaFree(d_cyc);
        cudaFree(d_sink);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    };
    // shared-memory bandwidth: one 1024-thread CTA per SM, 128 KiB read and written per round
    const int rounds = 200;
    const size_t smem = kSmemWords * sizeof(float4);
    ZQD_CUDA(cudaFuncSetAttribute(smem_bw_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    smem_bw_kernel<<<sms, 1024, smem>>>(rounds, d_cyc, d_sink); // warm-up
    ZQD_CUDA(cudaEventRecord(e0));
    smem_bw_kernel<<<sms, 1024, smem>>>(rounds, d_cyc, d_sink);
    ZQD_CUDA(cudaEventRecord(e1));
    ZQD_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    ZQD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    ZQD_CUDA(cudaMemcpy(cyc.data(), d_cyc, sms * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    unsigned long long cmax = 0;
    for (int i = 0; i < sms; ++i) cmax = std::max(cmax, cyc[i]);
    const double bytes_per_sm = 2.0 * (double)rounds * (double)smem; // read + write
    out->smem_bytes_per_cycle_per_sm = bytes_per_sm / (double)cmax;
    out->smem_gbs_per_sm = bytes_per_sm / (ms * 1e-3) / 1e9;
    // __syncthreads in a 256-thread CTA
    const int srounds = 20000;
    syncthreads_kernel<<<1, 256>>>(srounds, d_cyc, reinterpret_cast<int*>(d_sink));
    ZQD_CUDA(cudaMemcpy(cyc.data(), d_cyc, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    out->syncthreads_cycles = (double)cyc[0] / srounds;
    // barrier across a cluster of 16 CTAs (256 threads each)
    ZQD_CUDA(cudaFuncSetAttribute(cluster_barrier_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16, 1, 1);
    cfg.blockDim = dim3(256, 1, 1);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 16;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int crounds = 20000;
    ZQD_CUDA(cudaLaunchKernelEx(&cfg, cluster_barrier_kernel, crounds, d_cyc));
    ZQD_CUDA(cudaMemcpy(cyc.data(), d_cyc, 16 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    cmax = 0;
    for (int i = 0; i < 16; ++i) cmax = std::max(cmax, cyc[i]);
    out->cluster_barrier_cycles = (double)cmax / crounds;
    out->sm_clock_mhz = khz / 1000.0;
    out->sms = (uint32_t)sms;
    cleanup();
    return ZQD_OK;
}
