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
    const T c = (T)0.70710678118654752440084436210484903;
    // radix-2 split over j and j+4
    cx<T> b0 = add<T>(v[0], v[4]), b1 = add<T>(v[1], v[5]), b2 = add<T>(v[2], v[6]), b3 = add<T>(v[3], v[7]);
    cx<T> d0 = sub<T>(v[0], v[4]), d1 = sub<T>(v[1], v[5]), d2 = sub<T>(v[2], v[6]), d3 = sub<T>(v[3], v[7]);
    // d1 *= W, d2 *= W^2, d3 *= W^3 with W = exp(SIGN*2 pi i/8)
    if (SIGN < 0) {
        d1 = mk<T>(c * (d1.x + d1.y), c * (d1.y - d1.x));
        d3 = mk<T>(c * (d3.y - d3.x), -c * (d3.x + d3.y));
    } else {
        d1 = mk<T>(c * (d1.x - d1.y), c * (d1.x + d1.y));
        d3 = mk<T>(-c * (d3.x + d3.y), c * (d3.x - d3.y));
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
    const T c1 = (T)0.92387953251128675612818318939678829; // cos(pi/8)
    const T s1 = (T)0.38268343236508977172845998403039887; // sin(pi/8)
    const T h = (T)0.70710678118654752440084436210484903;
    cx<T> a[4][4];
#pragma unroll
    for (int j1 = 0; j1 < 4; ++j1) {
        cx<T> t[4] = {v[j1], v[j1 + 4], v[j1 + 8], v[j1 + 12]};
        dft4<SIGN, T>(t);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) a[j1][k2] = t[k2];
    }
    // twiddle a[j1][k2] *= w16^(j1*k2)
    const T cs[10] = {(T)1, c1, h, s1, (T)0, -s1, -h, -c1, (T)-1, -c1};
    const T sn[10] = {(T)0, s1, h, c1, (T)1, c1, h, s1, (T)0, -s1};
#pragma unroll
    for (int j1 = 1; j1 < 4; ++j1)
#pragma unroll
        for (int k2 = 1; k2 < 4; ++k2) {
            int e = j1 * k2; // 1..9
            cx<T> w = mk<T>(cs[e], SIGN < 0 ? -sn[e] : sn[e]);
            a[j1][k2] = mul<T>(a[j1][k2], w);
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
