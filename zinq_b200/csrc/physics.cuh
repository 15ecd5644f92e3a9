// physics.cuh -- per-grid-point physics shared by every propagation kernel:
// the diabatic potential V(r, t) (src/potential.zig:143-615), the FP64
// bytecode interpreter for `custom` expressions (replacing ExprTk,
// src/exprtk.cpp:32-40), and the FP64 symmetric eigensolver that replaces
// LAPACKE_dsyevd in eighBatch (src/linear_algebra.zig:28-70).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "expr.h"

namespace zqd {

constexpr int MAX_S = 4;
constexpr int MAX_D = 3;

enum PotKind : int { PK_HARMONIC = 0, PK_TIME_LINEAR, PK_TULLY_1, PK_TULLY_2, PK_TULLY_3, PK_CUSTOM, PK_LVC, PK_FILE };

// Device descriptor of a potential; pointers are device addresses.
struct PotDev {
    int kind, nd, ns, td;
    double prm[8];                 // harmonic k[nd]; time_linear a g; tully A B C D (E0)
    const uint32_t* code;          // custom: concatenated programs
    const double* consts;
    int code_off[MAX_S * MAX_S];   // program start of V[i*S+j]
    int const_off[MAX_S * MAX_S];
    const double* lvc;             // freq[nm] | exc[ns] | kappa[ns][nm] | lambda[ns][ns][nm]
    int lvc_nm;
    const double* file;            // nrow x ncol table
    int file_nrow, file_ncol, file_size;
};

__device__ __forceinline__ double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }

__device__ __forceinline__ double ipow_dev(double x, int e) {
    unsigned u = (unsigned)(e < 0 ? -e : e);
    double result = 1.0, base = x;
    bool first = true;
    while (u) {
        if (u & 1u) {
            result = first ? base : result * base;
            first = false;
        }
        u >>= 1;
        if (u) base = base * base;
    }
    return e < 0 ? 1.0 / result : result;
}

// Postfix interpreter of an ExprProgram (see expr.cpp for the instruction set).
static __device__ __noinline__ double vm_eval(const uint32_t* code, const double* consts, const double* r, double t) {
    double st[32];
    int sp = 0;
    for (int pc = 0; pc < 4096; ++pc) {
        uint32_t w = code[pc];
        int32_t a = arg_of(w);
        switch (op_of(w)) {
        case OP_END: return sp ? st[sp - 1] : nan("");
        case OP_CONST: st[sp++] = consts[a]; break;
        case OP_VAR: st[sp++] = r[a]; break;
        case OP_TIME: st[sp++] = t; break;
        case OP_NEG: st[sp - 1] = -st[sp - 1]; break;
        case OP_ADD: --sp; st[sp - 1] = __dadd_rn(st[sp - 1], st[sp]); break;
        case OP_SUB: --sp; st[sp - 1] = __dsub_rn(st[sp - 1], st[sp]); break;
        case OP_MUL: --sp; st[sp - 1] = __dmul_rn(st[sp - 1], st[sp]); break;
        case OP_DIV: --sp; st[sp - 1] = st[sp - 1] / st[sp]; break;
        case OP_MOD: --sp; st[sp - 1] = fmod(st[sp - 1], st[sp]); break;
        case OP_POW: --sp; st[sp - 1] = pow(st[sp - 1], st[sp]); break;
        case OP_IPOW: st[sp - 1] = ipow_dev(st[sp - 1], a); break;
        case OP_LT: --sp; st[sp - 1] = st[sp - 1] < st[sp] ? 1.0 : 0.0; break;
        case OP_LE: --sp; st[sp - 1] = st[sp - 1] <= st[sp] ? 1.0 : 0.0; break;
        case OP_GT: --sp; st[sp - 1] = st[sp - 1] > st[sp] ? 1.0 : 0.0; break;
        case OP_GE: --sp; st[sp - 1] = st[sp - 1] >= st[sp] ? 1.0 : 0.0; break;
        case OP_EQ: --sp; st[sp - 1] = st[sp - 1] == st[sp] ? 1.0 : 0.0; break;
        case OP_NE: --sp; st[sp - 1] = st[sp - 1] != st[sp] ? 1.0 : 0.0; break;
        case OP_IF: sp -= 2; st[sp - 1] = st[sp - 1] != 0.0 ? st[sp] : st[sp + 1]; break;
        case OP_MIN:
        case OP_MAX: {
            double v = st[sp - a];
            for (int i = 1; i < a; ++i) {
                double x = st[sp - a + i];
                v = op_of(w) == OP_MIN ? (x < v ? x : v) : (x > v ? x : v);
            }
            sp -= a - 1;
            st[sp - 1] = v;
            break;
        }
        case OP_FN2: {
            --sp;
            double x = st[sp - 1], y = st[sp];
            st[sp - 1] = a == F_ATAN2 ? atan2(x, y) : a == F_HYPOT ? hypot(x, y) : fmod(x, y);
            break;
        }
        case OP_FN1: {
            double x = st[sp - 1], v;
            switch (a) {
            case F_ABS: v = fabs(x); break;
            case F_SGN: v = sgn(x); break;
            case F_EXP: v = exp(x); break;
            case F_LOG: v = log(x); break;
            case F_LOG10: v = log10(x); break;
            case F_LOG2: v = log2(x); break;
            case F_SQRT: v = sqrt(x); break;
            case F_SIN: v = sin(x); break;
            case F_COS: v = cos(x); break;
            case F_TAN: v = tan(x); break;
            case F_ASIN: v = asin(x); break;
            case F_ACOS: v = acos(x); break;
            case F_ATAN: v = atan(x); break;
            case F_SINH: v = sinh(x); break;
            case F_COSH: v = cosh(x); break;
            case F_TANH: v = tanh(x); break;
            case F_ERF: v = erf(x); break;
            case F_ERFC: v = erfc(x); break;
            case F_FLOOR: v = floor(x); break;
            case F_CEIL: v = ceil(x); break;
            case F_ROUND: v = round(x); break;
            case F_TRUNC: v = trunc(x); break;
            case F_LOG1P: v = log1p(x); break;
            case F_EXPM1: v = expm1(x); break;
            default: v = cbrt(x); break;
            }
            st[sp - 1] = v;
            break;
        }
        default: return nan("");
        }
    }
    return nan("");
}

// Multilinear interpolation on a rectangular table (lerp, src/potential.zig:578-615).
static __device__ __noinline__ double file_lerp(const PotDev& P, int column, const double* r) {
    const int nr = P.nd;
    const int size = P.file_size;
    double result = 0;
    for (int i = 0; i < (1 << nr); ++i) {
        double w = 1;
        long long j = 0;
        long long stride = 1;
        for (int q = 0; q < nr - 1; ++q) stride *= size;
        for (int k = 0; k < nr; ++k) {
            int low = 0, high = size, mid = size / 2;
            while (low < high) {
                if (P.file[(long long)mid * stride * P.file_ncol + k] <= r[k]) low = mid + 1;
                else high = mid;
                mid = (low + high) / 2;
            }
            int idx = min(max(low, 1), size - 1);
            double x0 = P.file[(long long)(idx - 1) * stride * P.file_ncol + k];
            double x1 = P.file[(long long)idx * stride * P.file_ncol + k];
            double wgh = __dmul_rn(__dsub_rn(r[k], x0), 1.0 / __dsub_rn(x1, x0));
            bool upper = ((i >> (nr - k - 1)) & 1) == 1;
            double wm = upper ? wgh : __dsub_rn(1.0, wgh);
            w = __dmul_rn(w, wm);
            j += (long long)(upper ? idx : idx - 1) * stride;
            stride /= (size > 0 ? size : 1);
        }
        result = __dadd_rn(result, __dmul_rn(w, P.file[j * P.file_ncol + column]));
    }
    return result;
}

// V(r, t) as an S x S row-major matrix (Potential.eval, src/potential.zig:98-106).
// Products and sums are rounded separately, as the reference's Zig code does.
static __device__ __noinline__ void pot_eval(const PotDev& P, const double* r, double t, double* V) {
    switch (P.kind) {
    case PK_HARMONIC: { // :152-161
        double sum = 0;
        for (int i = 0; i < P.nd; ++i) sum = __dadd_rn(sum, __dmul_rn(__dmul_rn(r[i], r[i]), 0.5 * P.prm[i]));
        V[0] = sum;
        break;
    }
    case PK_TIME_LINEAR: { // :189-201
        double a = P.prm[0], g = P.prm[1];
        double v00 = __dmul_rn(__dsub_rn(t, a), a);
        V[0] = v00;
        V[1] = g;
        V[2] = g;
        V[3] = -v00;
        break;
    }
    case PK_TULLY_1: { // :231-247
        double A = P.prm[0], B = P.prm[1], C = P.prm[2], D = P.prm[3], x = r[0];
        double v00 = __dmul_rn(__dmul_rn(__dadd_rn(-exp(-__dmul_rn(fabs(x), B)), 1.0), A), sgn(x));
        double v01 = __dmul_rn(exp(-__dmul_rn(__dmul_rn(x, x), D)), C);
        V[0] = v00;
        V[1] = v01;
        V[2] = v01;
        V[3] = -v00;
        break;
    }
    case PK_TULLY_2: { // :279-297
        double A = P.prm[0], B = P.prm[1], C = P.prm[2], D = P.prm[3], E0 = P.prm[4], x = r[0];
        double v01 = __dmul_rn(exp(-__dmul_rn(__dmul_rn(x, x), D)), C);
        double v11 = __dadd_rn(-__dmul_rn(exp(-__dmul_rn(__dmul_rn(x, x), B)), A), E0);
        V[0] = 0.0;
        V[1] = v01;
        V[2] = v01;
        V[3] = v11;
        break;
    }
    case PK_TULLY_3: { // :329-344
        double A = P.prm[0], B = P.prm[1], C = P.prm[2], x = r[0];
        double v01 = __dmul_rn(__dadd_rn(__dmul_rn(__dsub_rn(1.0, exp(-__dmul_rn(fabs(x), C))), sgn(x)), 1.0), B);
        V[0] = A;
        V[1] = v01;
        V[2] = v01;
        V[3] = -A;
        break;
    }
    case PK_CUSTOM: // :409-412
        for (int e = 0; e < P.ns * P.ns; ++e) V[e] = vm_eval(P.code + P.code_off[e], P.consts + P.const_off[e], r, t);
        break;
    case PK_LVC: { // :523-558
        const double h = 6.62607015e-34, ec = 1.602176634e-19, c = 299792458.0, Eh = 4.3597447222060e-18;
        const double CM2EV = (1e2 * h * c) / ec, EV2AU = ec / Eh;
        const int nm = P.lvc_nm, ns = P.ns;
        const double* freq = P.lvc;
        const double* exc = freq + nm;
        const double* kap = exc + ns;
        const double* lmb = kap + ns * nm;
        double v0 = 0;
        for (int i = 0; i < nm; ++i) v0 = __dadd_rn(v0, __dmul_rn(__dmul_rn(r[i], r[i]), 0.5 * freq[i] * CM2EV));
        for (int n = 0; n < ns; ++n) {
            double term = exc[n];
            for (int i = 0; i < nm; ++i) term = __dadd_rn(term, __dmul_rn(r[i], kap[n * nm + i]));
            V[n * ns + n] = __dadd_rn(v0, term);
        }
        for (int m = 0; m < ns; ++m)
            for (int n = m + 1; n < ns; ++n) {
                double term = 0;
                for (int i = 0; i < nm; ++i) term = __dadd_rn(term, __dmul_rn(r[i], lmb[(m * ns + n) * nm + i]));
                V[m * ns + n] = term;
                V[n * ns + m] = term;
            }
        for (int i = 0; i < ns * ns; ++i) V[i] = __dmul_rn(V[i], EV2AU);
        break;
    }
    case PK_FILE: // :470-476
        for (int col = 0; col < P.ns * P.ns; ++col) V[col] = file_lerp(P, P.nd + col, r);
        break;
    }
}

// ------------------------------------------------------------------ eigh
// dlaev2 (LAPACK): eigensystem of [[a, b], [b, c]].
__device__ __forceinline__ void dlaev2_dev(double a, double b, double c, double& rt1, double& rt2, double& cs1,
                                           double& sn1) {
    double sm = __dadd_rn(a, c), df = __dsub_rn(a, c), adf = fabs(df), tb = __dadd_rn(b, b), ab = fabs(tb);
    double acmx, acmn, rt, cs, ct, tn;
    int sgn1, sgn2;
    if (fabs(a) > fabs(c)) {
        acmx = a;
        acmn = c;
    } else {
        acmx = c;
        acmn = a;
    }
    if (adf > ab) {
        double q = ab / adf;
        rt = __dmul_rn(adf, sqrt(__dadd_rn(1.0, __dmul_rn(q, q))));
    } else if (adf < ab) {
        double q = adf / ab;
        rt = __dmul_rn(ab, sqrt(__dadd_rn(1.0, __dmul_rn(q, q))));
    } else {
        rt = __dmul_rn(ab, 1.4142135623730950488016887242097);
    }
    if (sm < 0.0) {
        rt1 = __dmul_rn(0.5, __dsub_rn(sm, rt));
        sgn1 = -1;
        rt2 = __dsub_rn(__dmul_rn(acmx / rt1, acmn), __dmul_rn(b / rt1, b));
    } else if (sm > 0.0) {
        rt1 = __dmul_rn(0.5, __dadd_rn(sm, rt));
        sgn1 = 1;
        rt2 = __dsub_rn(__dmul_rn(acmx / rt1, acmn), __dmul_rn(b / rt1, b));
    } else {
        rt1 = __dmul_rn(0.5, rt);
        rt2 = __dmul_rn(-0.5, rt);
        sgn1 = 1;
    }
    if (df >= 0.0) {
        cs = __dadd_rn(df, rt);
        sgn2 = 1;
    } else {
        cs = __dsub_rn(df, rt);
        sgn2 = -1;
    }
    if (fabs(cs) > ab) {
        ct = -tb / cs;
        sn1 = 1.0 / sqrt(__dadd_rn(1.0, __dmul_rn(ct, ct)));
        cs1 = __dmul_rn(ct, sn1);
    } else if (ab == 0.0) {
        cs1 = 1.0;
        sn1 = 0.0;
    } else {
        tn = -cs / tb;
        cs1 = 1.0 / sqrt(__dadd_rn(1.0, __dmul_rn(tn, tn)));
        sn1 = __dmul_rn(tn, cs1);
    }
    if (sgn1 == sgn2) {
        tn = cs1;
        cs1 = -sn1;
        sn1 = tn;
    }
}

// dsyevd on a 2x2 matrix: the Householder reduction is the identity and dsteqr
// ends in dlaev2 plus one plane rotation, then a selection sort; so LAPACK's
// eigenvector signs are reproduced exactly.
__device__ __forceinline__ void eigh2_dev(const double* V, double* W, double* U) {
    const double eps = 1.1102230246251565404e-16, eps2 = eps * eps, safmin = 2.2250738585072014e-308;
    double d1 = V[0], d2 = V[3], e = V[1];
    double z11 = 1, z12 = 0, z21 = 0, z22 = 1;
    double tst = fabs(e);
    bool split = (tst == 0.0) || (tst <= __dmul_rn(__dmul_rn(sqrt(fabs(d1)), sqrt(fabs(d2))), eps));
    bool rotate = false;
    if (!split) {
        double anorm = fmax(fmax(fabs(d1), fabs(d2)), fabs(e));
        if (anorm != 0.0) {
            double t2 = __dmul_rn(fabs(e), fabs(e));
            if (fabs(d2) < fabs(d1))
                rotate = !(t2 <= __dadd_rn(__dmul_rn(__dmul_rn(eps2, fabs(d2)), fabs(d1)), safmin));
            else
                rotate = !(t2 <= __dadd_rn(__dmul_rn(__dmul_rn(eps2, fabs(d1)), fabs(d2)), safmin));
        }
    }
    if (rotate) {
        double rt1, rt2, c, s;
        dlaev2_dev(d1, e, d2, rt1, rt2, c, s);
        z11 = c;
        z21 = s;
        z12 = -s;
        z22 = c;
        d1 = rt1;
        d2 = rt2;
    }
    if (d2 < d1) {
        double t = d1;
        d1 = d2;
        d2 = t;
        t = z11;
        z11 = z12;
        z12 = t;
        t = z21;
        z21 = z22;
        z22 = t;
    }
    W[0] = d1;
    W[1] = d2;
    U[0] = z11;
    U[1] = z12;
    U[2] = z21;
    U[3] = z22;
}

// cyclic Jacobi for 3 <= n <= MAX_S; ascending, largest-|component| positive
template <int N> __device__ __noinline__ void eigh_jacobi_dev(const double* V, double* W, double* U) {
    double A[N * N], Z[N * N];
    for (int i = 0; i < N * N; ++i) {
        A[i] = V[i];
        Z[i] = 0;
    }
    for (int i = 0; i < N; ++i) Z[i * N + i] = 1;
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0, diag = 0;
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) {
                double a2 = __dmul_rn(A[i * N + j], A[i * N + j]);
                if (i != j) off = __dadd_rn(off, a2);
                else diag = __dadd_rn(diag, a2);
            }
        if (off <= 1e-36 * diag || off == 0.0) break;
        for (int p = 0; p < N - 1; ++p)
            for (int q = p + 1; q < N; ++q) {
                double apq = A[p * N + q];
                if (apq == 0.0) continue;
                double app = A[p * N + p], aqq = A[q * N + q];
                double theta = __dsub_rn(aqq, app) / __dmul_rn(2.0, apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / __dadd_rn(fabs(theta), sqrt(__dadd_rn(__dmul_rn(theta, theta), 1.0)));
                double c = 1.0 / sqrt(__dadd_rn(__dmul_rn(t, t), 1.0)), s = __dmul_rn(t, c);
                for (int k = 0; k < N; ++k) {
                    double akp = A[k * N + p], akq = A[k * N + q];
                    A[k * N + p] = __dsub_rn(__dmul_rn(c, akp), __dmul_rn(s, akq));
                    A[k * N + q] = __dadd_rn(__dmul_rn(s, akp), __dmul_rn(c, akq));
                }
                for (int k = 0; k < N; ++k) {
                    double apk = A[p * N + k], aqk = A[q * N + k];
                    A[p * N + k] = __dsub_rn(__dmul_rn(c, apk), __dmul_rn(s, aqk));
                    A[q * N + k] = __dadd_rn(__dmul_rn(s, apk), __dmul_rn(c, aqk));
                }
                for (int k = 0; k < N; ++k) {
                    double zkp = Z[k * N + p], zkq = Z[k * N + q];
                    Z[k * N + p] = __dsub_rn(__dmul_rn(c, zkp), __dmul_rn(s, zkq));
                    Z[k * N + q] = __dadd_rn(__dmul_rn(s, zkp), __dmul_rn(c, zkq));
                }
            }
    }
    double d[N];
    for (int i = 0; i < N; ++i) d[i] = A[i * N + i];
    for (int i = 0; i < N - 1; ++i) {
        int k = i;
        double p = d[i];
        for (int j = i + 1; j < N; ++j)
            if (d[j] < p) {
                k = j;
                p = d[j];
            }
        if (k != i) {
            d[k] = d[i];
            d[i] = p;
            for (int r = 0; r < N; ++r) {
                double t = Z[r * N + i];
                Z[r * N + i] = Z[r * N + k];
                Z[r * N + k] = t;
            }
        }
    }
    for (int m = 0; m < N; ++m) {
        int big = 0;
        for (int k = 1; k < N; ++k)
            if (fabs(Z[k * N + m]) > fabs(Z[big * N + m])) big = k;
        if (Z[big * N + m] < 0)
            for (int k = 0; k < N; ++k) Z[k * N + m] = -Z[k * N + m];
    }
    for (int i = 0; i < N; ++i) W[i] = d[i];
    for (int i = 0; i < N * N; ++i) U[i] = Z[i];
}

template <int S> __device__ __forceinline__ void eigh_dev(const double* V, double* W, double* U) {
    if constexpr (S == 1) {
        W[0] = V[0];
        U[0] = 1.0;
    } else if constexpr (S == 2) {
        eigh2_dev(V, W, U);
    } else {
        eigh_jacobi_dev<S>(V, W, U);
    }
}

// complex exponential with the special cases of std.math.complex.exp (musl cexp)
__device__ __forceinline__ void cexp_dev(double re, double im, double& ore, double& oim) {
    if (im == 0.0) {
        ore = exp(re);
        oim = im;
    } else if (re == 0.0) {
        sincos(im, &oim, &ore);
    } else {
        double e = exp(re), s, c;
        sincos(im, &s, &c);
        ore = __dmul_rn(e, c);
        oim = __dmul_rn(e, s);
    }
}

// Element (k, j) of R = U diag(exp(-i W dt / 2)) U^T * decay
// (Propagator.update, src/quantum_dynamics.zig:453-466).
template <int S>
__device__ __forceinline__ void propagator_entry(const double* W, const double* U, double dt_re, double dt_im, double decay,
                                                 int k, int j, double& out_re, double& out_im) {
    double sre = 0, sim = 0;
#pragma unroll
    for (int m = 0; m < S; ++m) {
        double ukm = U[k * S + m], ujm = U[j * S + m];
        // Complex(0, -0.5 W) * dt
        double a_im = -0.5 * W[m];
        double zre = __dsub_rn(__dmul_rn(0.0, dt_re), __dmul_rn(a_im, dt_im));
        double zim = __dadd_rn(__dmul_rn(0.0, dt_im), __dmul_rn(a_im, dt_re));
        double pre, pim;
        cexp_dev(zre, zim, pre, pim);
        sre = __dadd_rn(sre, __dmul_rn(__dmul_rn(pre, ukm), ujm));
        sim = __dadd_rn(sim, __dmul_rn(__dmul_rn(pim, ukm), ujm));
    }
    out_re = __dmul_rn(sre, decay);
    out_im = __dmul_rn(sim, decay);
}

} // namespace zqd
