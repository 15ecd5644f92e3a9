// spectrum.cu -- calcSpectrum (src/spectral_analysis.zig:13-44) on the device: Gaussian
// window of the autocorrelation, zero padding, a complex-to-real transform of length
// M = 2 (L + padding - 1) with FFTW's c2r conventions (Hermitian extension, the imaginary
// parts of X[0] and X[M/2] ignored, unnormalised, sign +1), the half swap and the dt scale.
// M is rarely a power of two, so the transform is evaluated directly: one thread per output,
// exact twiddles from the integer phase (k t) mod M, compensated FP64 sums.
#include <cmath>
#include <vector>

#include "cx.cuh"
#include "internal.h"

namespace zqd {

// acfpad[i] = acf[i] exp(-decay (i / L)^2) for i < L, zero up to lp
static __global__ void spec_window_kernel(const double* __restrict__ hist, int hc, int col, size_t L, size_t lp,
                                          double decay, double2* __restrict__ acfpad) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= lp) return;
    double2 z = make_double2(0.0, 0.0);
    if (i < L) {
        const double x = (double)i / (double)L;
        const double w = exp(-decay * x * x);
        z = make_double2(hist[i * hc + col] * w, hist[i * hc + col + 1] * w);
    }
    acfpad[i] = z;
}

// W[j] = exp(+2 pi i j / M)
static __global__ void spec_twiddle_kernel(size_t M, double2* __restrict__ W) {
    const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (j >= M) return;
    double s, c;
    sincospi(2.0 * (double)j / (double)M, &s, &c);
    W[j] = make_double2(c, s);
}

// sigma[t] = Re sum_k X~[k] exp(+2 pi i k t / M) over the Hermitian extension X~ of X[0..M/2],
// written to position (t + M/2) mod M and scaled by dt
static __global__ void spec_c2r_kernel(const double2* __restrict__ X, const double2* __restrict__ W, size_t M,
                                       double dt, double* __restrict__ sigma) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= M) return;
    const size_t h = M / 2;
    Acc acc;
    acc.add(X[0].x);
    acc.add((t & 1) ? -X[h].x : X[h].x);
    size_t j = t; // (k t) mod M for k = 1 (t < M)
    for (size_t k = 1; k < h; ++k) {
        const double2 w = W[j];
        acc.add(2.0 * (X[k].x * w.x - X[k].y * w.y));
        j += t;
        if (j >= M) j -= M;
    }
    sigma[t < h ? t + h : t - h] = acc.value() * dt;
}

// The spectrum of one solve from its device history (rows x hc, autocorrelation at column col).
int spectrum_device(cudaStream_t st, const double* d_hist, int hc, int col, size_t rows, const Opts& o, SolveOut& so,
                    uint64_t& d2h) {
    const size_t lp = rows + o.spectrum_padding;
    const size_t M = lp > 0 ? 2 * (lp - 1) : 0;
    so.acfpad.assign(2 * lp, 0.0);
    so.sigma.assign(M, 0.0);
    if (lp == 0) return ZQD_OK;
    double2 *acfpad = nullptr, *W = nullptr;
    double* sigma = nullptr;
    // pool blocks in the job's stream (cudaFree would wait for every stream of the device)
    auto cleanup = [&]() {
        dev_free(acfpad, st);
        dev_free(W, st);
        dev_free(sigma, st);
    };
    cudaError_t e = dev_alloc((void**)&acfpad, lp * sizeof(double2), st);
    if (e == cudaSuccess && M) e = dev_alloc((void**)&W, M * sizeof(double2), st);
    if (e == cudaSuccess && M) e = dev_alloc((void**)&sigma, M * sizeof(double), st);
    if (e != cudaSuccess) {
        cleanup();
        return fail(ZQD_ERR_DEVICE_OOM, std::string("spectrum buffers: ") + cudaGetErrorString(e));
    }
    const double decay = -std::log(o.spectrum_threshold);
    spec_window_kernel<<<(unsigned)((lp + 255) / 256), 256, 0, st>>>(d_hist, hc, col, rows, lp, decay, acfpad);
    if (M) {
        spec_twiddle_kernel<<<(unsigned)((M + 255) / 256), 256, 0, st>>>(M, W);
        spec_c2r_kernel<<<(unsigned)((M + 127) / 128), 128, 0, st>>>(acfpad, W, M, o.time_step, sigma);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(so.acfpad.data(), acfpad, lp * sizeof(double2), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && M) e = cudaMemcpyAsync(so.sigma.data(), sigma, M * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cleanup();
    if (e != cudaSuccess) return fail(ZQD_ERR_DEVICE, std::string("spectrum: ") + cudaGetErrorString(e));
    d2h += lp * sizeof(double2) + M * sizeof(double);
    return ZQD_OK;
}

} // namespace zqd
