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

// LAPACK dsyevd('V', 'U') for 3 <= n <= 4, as the reference's eighBatch calls it
// (src/linear_algebra.zig:55-70, LAPACKE_dsyevd row-major on a symmetric matrix), restated from the
// published netlib algorithm: dsytd2 (Householder reduction of the upper triangle, last column
// first), dsteqr('I') (implicit QL or QR, 2 x 2 blocks by dlaev2, selection sort) and dorm2l (the
// reflectors applied to the tridiagonal eigenvectors); so the eigenvector signs are LAPACK's.
// Every multiply and add is rounded on its own, in the published order.
namespace lapack_dev {
constexpr double EPS = 1.1102230246251565404e-16, SAFMIN = 2.2250738585072014e-308;
__device__ __forceinline__ double sgn(double a, double b) { return b >= 0 ? fabs(a) : -fabs(a); }
__device__ __forceinline__ double dlapy2(double x, double y) {
    const double xa = fabs(x), ya = fabs(y), w = fmax(xa, ya), z = fmin(xa, ya);
    if (z == 0.0 || w > 1.7976931348623157e308) return w;
    const double q = z / w;
    return __dmul_rn(w, sqrt(__dadd_rn(1.0, __dmul_rn(q, q))));
}
// dlartg (LAPACK >= 3.10): c >= 0, r carries the sign of f
__device__ __forceinline__ void dlartg(double f, double g, double& c, double& s, double& r) {
    const double rtmin = 1.4916681462400413e-154, rtmax = 4.740375954054589e153; // sqrt(safmin), sqrt(safmax/2)
    const double f1 = fabs(f), g1 = fabs(g);
    if (g == 0.0) {
        c = 1.0;
        s = 0.0;
        r = f;
    } else if (f == 0.0) {
        c = 0.0;
        s = sgn(1.0, g);
        r = g1;
    } else if (f1 > rtmin && f1 < rtmax && g1 > rtmin && g1 < rtmax) {
        const double d = sqrt(__dadd_rn(__dmul_rn(f, f), __dmul_rn(g, g)));
        c = f1 / d;
        r = sgn(d, f);
        s = g / r;
    } else {
        const double u = fmin(1.0 / SAFMIN, fmax(SAFMIN, fmax(f1, g1)));
        const double fs = f / u, gs = g / u, d = sqrt(__dadd_rn(__dmul_rn(fs, fs), __dmul_rn(gs, gs)));
        c = fabs(fs) / d;
        r = sgn(d, f);
        s = gs / r;
        r = __dmul_rn(r, u);
    }
}
// dlasr('R', 'V', forward or backward) on columns j0 .. j0+nc-1 of Z (N x N, row-major)
template <int N>
__device__ __forceinline__ void dlasr_rv(bool forward, int j0, int nc, const double* c, const double* s, double* Z) {
    for (int jj = 0; jj < nc - 1; ++jj) {
        const int j = forward ? jj : nc - 2 - jj;
        const double ct = c[j], st = s[j];
        if (ct == 1.0 && st == 0.0) continue;
        for (int i = 0; i < N; ++i) {
            const double t = Z[i * N + j0 + j + 1], a = Z[i * N + j0 + j];
            Z[i * N + j0 + j + 1] = __dsub_rn(__dmul_rn(ct, t), __dmul_rn(st, a));
            Z[i * N + j0 + j] = __dadd_rn(__dmul_rn(st, t), __dmul_rn(ct, a));
        }
    }
}
// dsteqr('I') on the tridiagonal (d, e); false if it did not converge in 30 n sweeps
template <int N> __device__ __noinline__ bool dsteqr(double* d, double* e, double* Z) {
    // sqrt(safmax) / 3 and sqrt(safmin) / eps^2, safmax = 1 / safmin
    const double eps2 = EPS * EPS, ssfmax = 6.703903964971299e153 / 3.0, ssfmin = 1.4916681462400413e-154 / eps2;
    for (int i = 0; i < N * N; ++i) Z[i] = 0.0;
    for (int i = 0; i < N; ++i) Z[i * N + i] = 1.0;
    double wc[N], ws[N];
    const int nmaxit = N * 30;
    int jtot = 0, l1 = 0;
    while (l1 <= N - 1) {
        if (l1 > 0) e[l1 - 1] = 0.0;
        int m = N - 1;
        for (int mm = l1; mm < N - 1; ++mm) {
            const double tst = fabs(e[mm]);
            if (tst == 0.0) {
                m = mm;
                break;
            }
            if (tst <= __dmul_rn(__dmul_rn(sqrt(fabs(d[mm])), sqrt(fabs(d[mm + 1]))), EPS)) {
                e[mm] = 0.0;
                m = mm;
                break;
            }
        }
        int l = l1;
        const int lsv = l, lendsv = m;
        int lend = m;
        l1 = m + 1;
        if (lend == l) continue;
        double anorm = 0.0;
        for (int i = l; i <= lend; ++i) anorm = fmax(anorm, fabs(d[i]));
        for (int i = l; i < lend; ++i) anorm = fmax(anorm, fabs(e[i]));
        if (anorm == 0.0) continue;
        double to = 0.0;
        if (anorm > ssfmax) to = ssfmax;
        if (anorm < ssfmin) to = ssfmin;
        if (to != 0.0) {
            for (int i = l; i <= lend; ++i) d[i] = __dmul_rn(d[i], to / anorm);
            for (int i = l; i < lend; ++i) e[i] = __dmul_rn(e[i], to / anorm);
        }
        if (fabs(d[lend]) < fabs(d[l])) {
            lend = lsv;
            l = lendsv;
        }
        if (lend > l) { // QL
            for (;;) {
                int mq = lend;
                for (int mm = l; mm < lend; ++mm) {
                    const double tst = __dmul_rn(fabs(e[mm]), fabs(e[mm]));
                    if (tst <= __dadd_rn(__dmul_rn(__dmul_rn(eps2, fabs(d[mm])), fabs(d[mm + 1])), SAFMIN)) {
                        mq = mm;
                        break;
                    }
                }
                if (mq < lend) e[mq] = 0.0;
                double p = d[l];
                if (mq == l) {
                    d[l] = p;
                    if (++l <= lend) continue;
                    break;
                }
                if (mq == l + 1) {
                    double rt1, rt2, c, s;
                    dlaev2_dev(d[l], e[l], d[l + 1], rt1, rt2, c, s);
                    wc[0] = c;
                    ws[0] = s;
                    dlasr_rv<N>(false, l, 2, wc, ws, Z);
                    d[l] = rt1;
                    d[l + 1] = rt2;
                    e[l] = 0.0;
                    l += 2;
                    if (l <= lend) continue;
                    break;
                }
                if (jtot == nmaxit) break;
                ++jtot;
                double g = __dsub_rn(d[l + 1], p) / __dmul_rn(2.0, e[l]);
                double r = dlapy2(g, 1.0);
                g = __dadd_rn(__dsub_rn(d[mq], p), e[l] / __dadd_rn(g, sgn(r, g)));
                double s = 1.0, c = 1.0;
                p = 0.0;
                for (int i = mq - 1; i >= l; --i) {
                    const double f = __dmul_rn(s, e[i]), b = __dmul_rn(c, e[i]);
                    dlartg(g, f, c, s, r);
                    if (i != mq - 1) e[i + 1] = r;
                    g = __dsub_rn(d[i + 1], p);
                    r = __dadd_rn(__dmul_rn(__dsub_rn(d[i], g), s), __dmul_rn(__dmul_rn(2.0, c), b));
                    p = __dmul_rn(s, r);
                    d[i + 1] = __dadd_rn(g, p);
                    g = __dsub_rn(__dmul_rn(c, r), b);
                    wc[i - l] = c;
                    ws[i - l] = -s;
                }
                dlasr_rv<N>(false, l, mq - l + 1, wc, ws, Z);
                d[l] = __dsub_rn(d[l], p);
                e[l] = g;
            }
        } else { // QR
            for (;;) {
                int mq = lend;
                for (int mm = l; mm > lend; --mm) {
                    const double tst = __dmul_rn(fabs(e[mm - 1]), fabs(e[mm - 1]));
                    if (tst <= __dadd_rn(__dmul_rn(__dmul_rn(eps2, fabs(d[mm])), fabs(d[mm - 1])), SAFMIN)) {
                        mq = mm;
                        break;
                    }
                }
                if (mq > lend) e[mq - 1] = 0.0;
                double p = d[l];
                if (mq == l) {
                    d[l] = p;
                    if (--l >= lend) continue;
                    break;
                }
                if (mq == l - 1) {
                    double rt1, rt2, c, s;
                    dlaev2_dev(d[l - 1], e[l - 1], d[l], rt1, rt2, c, s);
                    wc[0] = c;
                    ws[0] = s;
                    dlasr_rv<N>(true, l - 1, 2, wc, ws, Z);
                    d[l - 1] = rt1;
                    d[l] = rt2;
                    e[l - 1] = 0.0;
                    l -= 2;
                    if (l >= lend) continue;
                    break;
                }
                if (jtot == nmaxit) break;
                ++jtot;
                double g = __dsub_rn(d[l - 1], p) / __dmul_rn(2.0, e[l - 1]);
                double r = dlapy2(g, 1.0);
                g = __dadd_rn(__dsub_rn(d[mq], p), e[l - 1] / __dadd_rn(g, sgn(r, g)));
                double s = 1.0, c = 1.0;
                p = 0.0;
                for (int i = mq; i <= l - 1; ++i) {
                    const double f = __dmul_rn(s, e[i]), b = __dmul_rn(c, e[i]);
                    dlartg(g, f, c, s, r);
                    if (i != mq) e[i - 1] = r;
                    g = __dsub_rn(d[i], p);
                    r = __dadd_rn(__dmul_rn(__dsub_rn(d[i + 1], g), s), __dmul_rn(__dmul_rn(2.0, c), b));
                    p = __dmul_rn(s, r);
                    d[i] = __dadd_rn(g, p);
                    g = __dsub_rn(__dmul_rn(c, r), b);
                    wc[i - mq] = c;
                    ws[i - mq] = s;
                }
                dlasr_rv<N>(true, mq, l - mq + 1, wc, ws, Z);
                d[l] = __dsub_rn(d[l], p);
                e[l - 1] = g;
            }
        }
        if (to != 0.0) {
            for (int i = lsv; i <= lendsv; ++i) d[i] = __dmul_rn(d[i], anorm / to);
            for (int i = lsv; i < lendsv; ++i) e[i] = __dmul_rn(e[i], anorm / to);
        }
        if (jtot >= nmaxit) return false;
    }
    for (int ii = 1; ii < N; ++ii) { // selection sort, ascending, swapping eigenvectors
        const int i = ii - 1;
        int k = i;
        double p = d[i];
        for (int j = ii; j < N; ++j)
            if (d[j] < p) {
                k = j;
                p = d[j];
            }
        if (k != i) {
            d[k] = d[i];
            d[i] = p;
            for (int r = 0; r < N; ++r) {
                const double t = Z[r * N + i];
                Z[r * N + i] = Z[r * N + k];
                Z[r * N + k] = t;
            }
        }
    }
    return true;
}
} // namespace lapack_dev

// dsyevd('V', 'U') of the symmetric N x N matrix V (row-major, upper triangle read); W ascending,
// U[k*N + m] = component k of eigenvector m.  A non-converged case (never seen) leaves NaN.
template <int N> __device__ __noinline__ void eigh_lapack_dev(const double* V, double* W, double* U) {
    using namespace lapack_dev;
    double A[N][N], d[N], e[N], tau[N];
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) A[i][j] = V[i * N + j];
    for (int i = N - 1; i >= 1; --i) { // dsytd2('U')
        double alpha = A[i - 1][i], taui = 0.0;
        if (i > 1) { // dlarfg(i, A(i, i+1), A(1:i-1, i+1))
            // dnrm2 scaled by the largest magnitude: tiny couplings must not underflow to denormals
            double big = 0.0;
            for (int k = 0; k < i - 1; ++k) big = fmax(big, fabs(A[k][i]));
            double xn = 0.0;
            if (big > 0.0) {
                double ssq = 0.0;
                for (int k = 0; k < i - 1; ++k) {
                    const double q = A[k][i] / big;
                    ssq = __dadd_rn(ssq, __dmul_rn(q, q));
                }
                xn = __dmul_rn(big, sqrt(ssq));
            }
            if (xn != 0.0) {
                double beta = -sgn(dlapy2(alpha, xn), alpha);
                // dlarfg's rescaling: while |beta| < safmin / eps, scale x and alpha by eps / safmin
                const double sfmin = SAFMIN / EPS, rsafmn = 1.0 / sfmin;
                int knt = 0;
                if (fabs(beta) < sfmin) {
                    do {
                        ++knt;
                        for (int k = 0; k < i - 1; ++k) A[k][i] = __dmul_rn(A[k][i], rsafmn);
                        beta = __dmul_rn(beta, rsafmn);
                        alpha = __dmul_rn(alpha, rsafmn);
                    } while (fabs(beta) < sfmin && knt < 20);
                    double big2 = 0.0, ssq = 0.0;
                    for (int k = 0; k < i - 1; ++k) big2 = fmax(big2, fabs(A[k][i]));
                    for (int k = 0; k < i - 1; ++k) {
                        const double q = A[k][i] / big2;
                        ssq = __dadd_rn(ssq, __dmul_rn(q, q));
                    }
                    beta = -sgn(dlapy2(alpha, __dmul_rn(big2, sqrt(ssq))), alpha);
                }
                taui = __dsub_rn(beta, alpha) / beta;
                const double sc = 1.0 / __dsub_rn(alpha, beta);
                for (int k = 0; k < i - 1; ++k) A[k][i] = __dmul_rn(A[k][i], sc);
                for (int j = 0; j < knt; ++j) beta = __dmul_rn(beta, sfmin);
                alpha = beta;
            }
        }
        A[i - 1][i] = alpha;
        e[i - 1] = alpha;
        if (taui != 0.0) {
            A[i - 1][i] = 1.0;
            double y[N];
            for (int k = 0; k < N; ++k) y[k] = 0.0;
            for (int j = 0; j < i; ++j) { // dsymv('U'): y = taui A v
                const double t1 = __dmul_rn(taui, A[j][i]);
                double t2 = 0.0;
                for (int k = 0; k < j; ++k) {
                    y[k] = __dadd_rn(y[k], __dmul_rn(t1, A[k][j]));
                    t2 = __dadd_rn(t2, __dmul_rn(A[k][j], A[k][i]));
                }
                y[j] = __dadd_rn(y[j], __dadd_rn(__dmul_rn(t1, A[j][j]), __dmul_rn(taui, t2)));
            }
            double dot = 0.0;
            for (int k = 0; k < i; ++k) dot = __dadd_rn(dot, __dmul_rn(y[k], A[k][i]));
            const double al = __dmul_rn(__dmul_rn(-0.5, taui), dot);
            for (int k = 0; k < i; ++k) y[k] = __dadd_rn(y[k], __dmul_rn(al, A[k][i]));
            for (int j = 0; j < i; ++j) // dsyr2('U'): A -= v w' + w v'
                if (A[j][i] != 0.0 || y[j] != 0.0) {
                    const double t1 = -y[j], t2 = -A[j][i];
                    for (int k = 0; k <= j; ++k)
                        A[k][j] = __dadd_rn(A[k][j], __dadd_rn(__dmul_rn(A[k][i], t1), __dmul_rn(y[k], t2)));
                }
            A[i - 1][i] = e[i - 1];
        }
        d[i] = A[i][i];
        tau[i - 1] = taui;
    }
    d[0] = A[0][0];
    double Z[N * N];
    if (!dsteqr<N>(d, e, Z)) {
        for (int i = 0; i < N; ++i) W[i] = nan("");
        for (int i = 0; i < N * N; ++i) U[i] = nan("");
        return;
    }
    for (int i = 1; i <= N - 1; ++i) { // dorm2l('L', 'N'): Z(1:i, :) <- H(i) Z(1:i, :)
        const double t = tau[i - 1];
        if (t == 0.0) continue;
        double v[N];
        for (int k = 0; k < i - 1; ++k) v[k] = A[k][i];
        v[i - 1] = 1.0;
        for (int c = 0; c < N; ++c) {
            double w = 0.0;
            for (int k = 0; k < i; ++k) w = __dadd_rn(w, __dmul_rn(Z[k * N + c], v[k]));
            for (int k = 0; k < i; ++k) Z[k * N + c] = __dsub_rn(Z[k * N + c], __dmul_rn(__dmul_rn(t, v[k]), w));
        }
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
        eigh_lapack_dev<S>(V, W, U);
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
