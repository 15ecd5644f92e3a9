// cx.cuh -- complex arithmetic and register-resident small DFTs for the
// split-operator kernels (sm_100a).  Complex values are interleaved (re, im)
// pairs held in double2 / float2 so that one element moves as one 16- or
// 8-byte access, matching the reference's Matrix(Complex(f64)) layout
// (src/wavepacket.zig:175, src/tensor.zig:8-149).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace zqd {

template <typename T> struct cx_t;
template <> struct cx_t<double> { using type = double2; };
template <> struct cx_t<float> { using type = float2; };
template <typename T> using cx = typename cx_t<T>::type;

template <typename T> __host__ __device__ __forceinline__ cx<T> mk(T re, T im) {
    cx<T> z;
    z.x = re;
    z.y = im;
    return z;
}
template <typename T> __device__ __forceinline__ cx<T> add(cx<T> a, cx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ cx<T> sub(cx<T> a, cx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
// (a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re): std.math.Complex.mul order
template <typename T> __device__ __forceinline__ cx<T> mul(cx<T> a, cx<T> b) {
    return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __device__ __forceinline__ cx<T> conj(cx<T> a) { return mk<T>(a.x, -a.y); }
template <typename T> __device__ __forceinline__ cx<T> scale(cx<T> a, T s) { return mk<T>(a.x * s, a.y * s); }
// multiply by -i (SIGN = -1) or +i (SIGN = +1)
template <int SIGN, typename T> __device__ __forceinline__ cx<T> mul_i(cx<T> a) {
    return SIGN < 0 ? mk<T>(a.y, -a.x) : mk<T>(-a.y, a.x);
}
// twiddle w with the direction applied: forward tables hold exp(-2 pi i t / n)
template <int SIGN, typename T> __device__ __forceinline__ cx<T> twiddle(cx<T> w) { return SIGN < 0 ? w : conj<T>(w); }

template <typename T> __device__ __forceinline__ T sqmag(cx<T> a) { return a.x * a.x + a.y * a.y; }

// ------------------------------------------------------------ phase tables
// Entries of twiddle and phase tables.  FP64: one double2.  FP32: an
// unevaluated pair hi + lo of float2 (packed in a float4), split from the
// FP64 value, so a table entry carries ~FP64 accuracy while every multiply
// stays in FP32 arithmetic.  A single rounded float would make each step's
// phase error identical and the error would grow linearly with the number
// of steps; with the pair only the (sign-varying) product rounding remains.
template <typename T> struct tab_t;
template <> struct tab_t<double> { using type = double2; };
template <> struct tab_t<float> { using type = float4; };
template <typename T> using Tab = typename tab_t<T>::type;

template <typename T> __host__ __device__ inline Tab<T> mktab(double re, double im);
template <> __host__ __device__ inline double2 mktab<double>(double re, double im) {
    double2 w;
    w.x = re;
    w.y = im;
    return w;
}
template <> __host__ __device__ inline float4 mktab<float>(double re, double im) {
    float4 w;
    w.x = (float)re;
    w.y = (float)im;
    w.z = (float)(re - (double)w.x);
    w.w = (float)(im - (double)w.y);
    return w;
}

// a * w (SIGN < 0) or a * conj(w) (SIGN > 0)
template <int SIGN> __device__ __forceinline__ double2 tmul(double2 a, double2 w) {
    return mul<double>(a, twiddle<SIGN, double>(w));
}
template <int SIGN> __device__ __forceinline__ float2 tmul(float2 a, float4 w) {
    const float hx = w.x, hy = SIGN < 0 ? w.y : -w.y, lx = w.z, ly = SIGN < 0 ? w.w : -w.w;
    const float tre = fmaf(a.x, lx, -a.y * ly), tim = fmaf(a.x, ly, a.y * lx);
    float2 r;
    r.x = fmaf(a.x, hx, fmaf(-a.y, hy, tre));
    r.y = fmaf(a.x, hy, fmaf(a.y, hx, tim));
    return r;
}

// x * sqrt(1/2): FP32 carries the constant as hi + lo as well
__device__ __forceinline__ double mul_rsqrt2(double x) { return x * 0.70710678118654752440084436210484903; }
__device__ __forceinline__ float mul_rsqrt2(float x) { return fmaf(0.70710677f, x, 1.21016175e-08f * x); }

// ------------------------------------------------------------ small DFTs
// In-register DFTs of length 2, 4, 8, 16 (natural order in and out).
// SIGN -1: X[k] = sum x[j] exp(-2 pi i jk/R); SIGN +1 the conjugate kernel.
template <int SIGN, typename T> __device__ __forceinline__ void dft2(cx<T>* v) {
    cx<T> a = v[0], b = v[1];
    v[0] = add<T>(a, b);
    v[1] = sub<T>(a, b);
}

template <int SIGN, typename T> __device__ __forceinline__ void dft4(cx<T>* v) {
    cx<T> s02 = add<T>(v[0], v[2]), d02 = sub<T>(v[0], v[2]);
    cx<T> s13 = add<T>(v[1], v[3]), d13 = mul_i<SIGN, T>(sub<T>(v[1], v[3]));
    v[0] = add<T>(s02, s13);
    v[2] = sub<T>(s02, s13);
    v[1] = add<T>(d02, d13);
    v[3] = sub<T>(d02, d13);
}

template <int SIGN, typename T> __device__ __forceinline__ void dft8(cx<T>* v) {
    // radix-2 split over j and j+4
    cx<T> b0 = add<T>(v[0], v[4]), b1 = add<T>(v[1], v[5]), b2 = add<T>(v[2], v[6]), b3 = add<T>(v[3], v[7]);
    cx<T> d0 = sub<T>(v[0], v[4]), d1 = sub<T>(v[1], v[5]), d2 = sub<T>(v[2], v[6]), d3 = sub<T>(v[3], v[7]);
    // d1 *= W, d2 *= W^2, d3 *= W^3 with W = exp(SIGN*2 pi i/8)
    if (SIGN < 0) {
        d1 = mk<T>(mul_rsqrt2(d1.x + d1.y), mul_rsqrt2(d1.y - d1.x));
        d3 = mk<T>(mul_rsqrt2(d3.y - d3.x), -mul_rsqrt2(d3.x + d3.y));
    } else {
        d1 = mk<T>(mul_rsqrt2(d1.x - d1.y), mul_rsqrt2(d1.x + d1.y));
        d3 = mk<T>(-mul_rsqrt2(d3.x + d3.y), mul_rsqrt2(d3.x - d3.y));
    }
    d2 = mul_i<SIGN, T>(d2);
    // two 4-point DFTs
    cx<T> s02 = add<T>(b0, b2), e02 = sub<T>(b0, b2), s13 = add<T>(b1, b3), e13 = mul_i<SIGN, T>(sub<T>(b1, b3));
    v[0] = add<T>(s02, s13);
    v[4] = sub<T>(s02, s13);
    v[2] = add<T>(e02, e13);
    v[6] = sub<T>(e02, e13);
    cx<T> t02 = add<T>(d0, d2), f02 = sub<T>(d0, d2), t13 = add<T>(d1, d3), f13 = mul_i<SIGN, T>(sub<T>(d1, d3));
    v[1] = add<T>(t02, t13);
    v[5] = sub<T>(t02, t13);
    v[3] = add<T>(f02, f13);
    v[7] = sub<T>(f02, f13);
}

// 16 = 4 x 4: column DFTs, twiddles exp(SIGN 2 pi i j1 k2 / 16), row DFTs, transpose
template <int SIGN, typename T> __device__ __forceinline__ void dft16(cx<T>* v) {
    const double c1 = 0.92387953251128675612818318939678829; // cos(pi/8)
    const double s1 = 0.38268343236508977172845998403039887; // sin(pi/8)
    const double h = 0.70710678118654752440084436210484903;
    cx<T> a[4][4];
#pragma unroll
    for (int j1 = 0; j1 < 4; ++j1) {
        cx<T> t[4] = {v[j1], v[j1 + 4], v[j1 + 8], v[j1 + 12]};
        dft4<SIGN, T>(t);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) a[j1][k2] = t[k2];
    }
    // twiddle a[j1][k2] *= w16^(j1*k2); table entries exp(-2 pi i e/16), conjugated for SIGN > 0
    const double cs[10] = {1, c1, h, s1, 0, -s1, -h, -c1, -1, -c1};
    const double sn[10] = {0, s1, h, c1, 1, c1, h, s1, 0, -s1};
#pragma unroll
    for (int j1 = 1; j1 < 4; ++j1)
#pragma unroll
        for (int k2 = 1; k2 < 4; ++k2) {
            const int e = j1 * k2; // 1..9
            a[j1][k2] = tmul<SIGN>(a[j1][k2], mktab<T>(cs[e], -sn[e]));
        }
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
        cx<T> t[4] = {a[0][k2], a[1][k2], a[2][k2], a[3][k2]};
        dft4<SIGN, T>(t);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) v[k2 + 4 * k1] = t[k1];
    }
}

template <int R, int SIGN, typename T> __device__ __forceinline__ void dft(cx<T>* v) {
    if constexpr (R == 1) {
    } else if constexpr (R == 2) {
        dft2<SIGN, T>(v);
    } else if constexpr (R == 4) {
        dft4<SIGN, T>(v);
    } else if constexpr (R == 8) {
        dft8<SIGN, T>(v);
    } else if constexpr (R == 16) {
        dft16<SIGN, T>(v);
    }
}

// ---------------------------------------------------- compensated sums
// Neumaier summation in FP64: every observable accumulates through this.
struct Acc {
    double s, c;
    __host__ __device__ __forceinline__ Acc() : s(0.0), c(0.0) {}
    __host__ __device__ __forceinline__ void add(double x) {
        double t = s + x;
        if (fabs(s) >= fabs(x))
            c += (s - t) + x;
        else
            c += (x - t) + s;
        s = t;
    }
    __host__ __device__ __forceinline__ double value() const { return s + c; }
};

} // namespace zqd
