// fft_seam.cu -- stand-alone N-D complex FFT of a device buffer (the FftPlan
// seam, src/fourier_transform.zig:8-49).  Each CTA stages one line of one axis
// in shared memory, runs the Stockham passes of the propagator kernels and
// writes it back; the inverse applies the reference's 1/N afterwards.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"
#include "line_kernel.cuh"

using namespace zqd;

struct zqd_fft {
    int ndim = 1, n = 0, sign = -1, logn = 0;
    size_t N = 0;
    bool fp32 = false;
    void* tw = nullptr;
    ~zqd_fft() {
        if (tw) cudaFree(tw);
    }
};

template <typename T, int SIGN>
__global__ void __launch_bounds__(512) fft_axis_kernel(cx<T>* data, int n, int logn, size_t stride, size_t N,
                                                       const Tab<T>* tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* buf = reinterpret_cast<cx<T>*>(smem_raw);
    const size_t line = blockIdx.x; // line index among N / n
    const size_t outer = line / stride, inner = line % stride;
    const size_t base = outer * stride * n + inner;
    for (int i = threadIdx.x; i < n; i += blockDim.x) buf[padx<T>(i)] = data[base + (size_t)i * stride];
    __syncthreads();
    fft_local<T, SIGN, 16>(buf, padded_len<T>(n), logn, 1, tw, 1);
    for (int i = threadIdx.x; i < n; i += blockDim.x) data[base + (size_t)i * stride] = buf[padx<T>(i)];
}

template <typename T> __global__ void scale_kernel(cx<T>* data, size_t N, double s) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < N) data[i] = mk<T>((T)((double)data[i].x / (1.0 / s)), (T)((double)data[i].y / (1.0 / s)));
}

extern "C" int zqd_fft_plan_create(uint32_t ndim, const int* shape, int sign, zqd_precision precision, zqd_fft** out) {
    if (!out || !shape) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    *out = nullptr;
    if (ndim == 0 || ndim > 3) return fail(ZQD_ERR_PLAN_FAILED, "FFT RANK MUST BE 1..3");
    for (uint32_t i = 1; i < ndim; ++i)
        if (shape[i] != shape[0]) return fail(ZQD_ERR_PLAN_FAILED, "FFT SHAPE MUST BE n^ndim");
    int n = shape[0];
    if (n < 2 || (n & (n - 1)) || n > 8192) return fail(ZQD_ERR_PLAN_FAILED, "FFT LENGTH MUST BE A POWER OF TWO 2..8192");
    if (sign != -1 && sign != 1) return fail(ZQD_ERR_PLAN_FAILED, "FFT SIGN MUST BE -1 OR +1");
    if (precision != ZQD_FP64 && precision != ZQD_FP32_MIXED)
        return fail(ZQD_ERR_INVALID_INPUT, "FFT PRECISION MUST BE ZQD_FP64 OR ZQD_FP32_MIXED");
    std::unique_ptr<zqd_fft> p(new zqd_fft());
    p->ndim = (int)ndim;
    p->n = n;
    p->sign = sign;
    while ((1 << p->logn) < n) ++p->logn;
    p->N = 1;
    for (uint32_t i = 0; i < ndim; ++i) p->N *= (size_t)n;
    p->fp32 = precision == ZQD_FP32_MIXED;
    std::vector<double> tw = twiddles_f64(n);
    if (p->fp32) {
        std::vector<float4> f(n);
        for (int t = 0; t < n; ++t) f[t] = mktab<float>(tw[2 * t], tw[2 * t + 1]);
        ZQD_CUDA(cudaMalloc(&p->tw, f.size() * sizeof(float4)));
        ZQD_CUDA(cudaMemcpy(p->tw, f.data(), f.size() * sizeof(float4), cudaMemcpyHostToDevice));
    } else {
        ZQD_CUDA(cudaMalloc(&p->tw, tw.size() * sizeof(double)));
        ZQD_CUDA(cudaMemcpy(p->tw, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    *out = p.release();
    return ZQD_OK;
}

template <typename T> static int fft_exec(zqd_fft* p, void* data, cudaStream_t st) {
    const int threads = std::max(32, std::min(512, ((p->n / 16) + 31) / 32 * 32));
    const size_t smem = (size_t)padded_len<T>(p->n) * sizeof(cx<T>);
    auto kf = fft_axis_kernel<T, -1>;
    auto ki = fft_axis_kernel<T, 1>;
    ZQD_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ZQD_CUDA(cudaFuncSetAttribute(ki, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    size_t stride = 1;
    for (int a = p->ndim - 1; a >= 0; --a) {
        unsigned lines = (unsigned)(p->N / p->n);
        if (p->sign < 0)
            kf<<<lines, threads, smem, st>>>((cx<T>*)data, p->n, p->logn, stride, p->N, (const Tab<T>*)p->tw);
        else
            ki<<<lines, threads, smem, st>>>((cx<T>*)data, p->n, p->logn, stride, p->N, (const Tab<T>*)p->tw);
        ZQD_CUDA(cudaGetLastError());
        stride *= (size_t)p->n;
    }
    if (p->sign > 0) {
        scale_kernel<T><<<(unsigned)((p->N + 255) / 256), 256, 0, st>>>((cx<T>*)data, p->N, 1.0 / (double)p->N);
        ZQD_CUDA(cudaGetLastError());
    }
    return ZQD_OK;
}

extern "C" int zqd_fft_execute(zqd_fft* p, void* data, void* stream) {
    if (!p || !data) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    cudaStream_t st = (cudaStream_t)stream;
    return p->fp32 ? fft_exec<float>(p, data, st) : fft_exec<double>(p, data, st);
}

extern "C" void zqd_fft_destroy(zqd_fft* p) { delete p; }

// ------------------------------------------------------------ no-allocation variant
// For callers that cannot allocate device memory (code running under an
// allocator it must not bypass, or a host that only owns a fixed arena): the
// twiddle table the transform needs lives in this file-scope array instead of
// a cudaMalloc'ed plan buffer.  128 KiB (8192 entries of 16 bytes, enough for
// FP64 pairs and FP32 hi/lo quadruples) stays resident on every GPU that loads
// the library until the process exits.
constexpr int ZQD_NOALLOC_FFT_MAX_N = 8192;
static __device__ __align__(256) double2 g_noalloc_twiddles[ZQD_NOALLOC_FFT_MAX_N];

// exp(-2 pi i t / n) computed on the device with sincospi (no host copy)
template <typename T> __global__ void noalloc_twiddle_kernel(Tab<T>* tw, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double s, c;
    sincospi(2.0 * (double)t / (double)n, &s, &c);
    tw[t] = mktab<T>(c, -s);
}

template <typename T>
static int fft_noalloc_exec(int ndim, int n, int logn, size_t N, int sign, Tab<T>* tw, void* data, cudaStream_t st) {
    noalloc_twiddle_kernel<T><<<(n + 127) / 128, 128, 0, st>>>(tw, n);
    ZQD_CUDA(cudaGetLastError());
    const int threads = std::max(32, std::min(512, ((n / 16) + 31) / 32 * 32));
    const size_t smem = (size_t)padded_len<T>(n) * sizeof(cx<T>);
    auto kf = fft_axis_kernel<T, -1>;
    auto ki = fft_axis_kernel<T, 1>;
    ZQD_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ZQD_CUDA(cudaFuncSetAttribute(ki, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    size_t stride = 1;
    for (int a = ndim - 1; a >= 0; --a) {
        const unsigned lines = (unsigned)(N / n);
        if (sign < 0) kf<<<lines, threads, smem, st>>>((cx<T>*)data, n, logn, stride, N, tw);
        else ki<<<lines, threads, smem, st>>>((cx<T>*)data, n, logn, stride, N, tw);
        ZQD_CUDA(cudaGetLastError());
        stride *= (size_t)n;
    }
    if (sign > 0) {
        scale_kernel<T><<<(unsigned)((N + 255) / 256), 256, 0, st>>>((cx<T>*)data, N, 1.0 / (double)N);
        ZQD_CUDA(cudaGetLastError());
    }
    return ZQD_OK;
}

extern "C" int zqd_fft_execute_noalloc(uint32_t ndim, const int* shape, int sign, zqd_precision precision,
                                       void* device_inout, void* cuda_stream) {
    if (!shape || !device_inout) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (ndim == 0 || ndim > 3) return fail(ZQD_ERR_PLAN_FAILED, "FFT RANK MUST BE 1..3");
    for (uint32_t i = 1; i < ndim; ++i)
        if (shape[i] != shape[0]) return fail(ZQD_ERR_PLAN_FAILED, "FFT SHAPE MUST BE n^ndim");
    const int n = shape[0];
    if (n > ZQD_NOALLOC_FFT_MAX_N)
        return fail(ZQD_ERR_UNSUPPORTED, "FFT LENGTH " + std::to_string(n) + " EXCEEDS THE 8192-POINT STATIC TWIDDLE "
                                         "TABLE OF zqd_fft_execute_noalloc");
    if (n < 2 || (n & (n - 1))) return fail(ZQD_ERR_PLAN_FAILED, "FFT LENGTH MUST BE A POWER OF TWO 2..8192");
    if (sign != -1 && sign != 1) return fail(ZQD_ERR_PLAN_FAILED, "FFT SIGN MUST BE -1 OR +1");
    if (precision != ZQD_FP64 && precision != ZQD_FP32_MIXED)
        return fail(ZQD_ERR_INVALID_INPUT, "FFT PRECISION MUST BE ZQD_FP64 OR ZQD_FP32_MIXED");
    // device address of the static table, looked up once per device with that device current
    static std::mutex mu;
    static void* table[64] = {};
    int dev = 0;
    ZQD_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(ZQD_ERR_UNSUPPORTED, "DEVICE ORDINAL ABOVE 63");
    void* tw = nullptr;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!table[dev]) {
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_twiddles);
            if (e != cudaSuccess) return fail(ZQD_ERR_DEVICE, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            table[dev] = ptr;
        }
        tw = table[dev];
    }
    int logn = 0;
    while ((1 << logn) < n) ++logn;
    size_t N = 1;
    for (uint32_t i = 0; i < ndim; ++i) N *= (size_t)n;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    return precision == ZQD_FP32_MIXED
               ? fft_noalloc_exec<float>((int)ndim, n, logn, N, sign, (Tab<float>*)tw, device_inout, st)
               : fft_noalloc_exec<double>((int)ndim, n, logn, N, sign, (Tab<double>*)tw, device_inout, st);
}
