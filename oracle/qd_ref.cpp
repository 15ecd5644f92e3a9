// qd_ref.cpp -- TEST INFRASTRUCTURE ONLY: the oracle.
//
// A single-threaded-by-default CPU restatement, in FP64, of Zinq's grid
// split-operator quantum-dynamics path (tjira/zinq).  Each function cites the
// reference file:line whose arithmetic it follows.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline legs load it; the CUDA
// product never links or calls it.
//
// Conventions fixed here (the reference delegates them to third-party code
// that is not present in this tree):
//   * FFT: own radix-2 decimation-in-time transform with twiddles computed in
//     long double and rounded (FFTW 3.3.11 in the reference,
//     src/fourier_transform.zig:38-47); Bluestein for other lengths.
//     Forward sign -1 unnormalised, inverse sign +1 followed by a 1/N loop.
//   * eigh: restates LAPACK dsyevd('V', 'U') (OpenBLAS 0.3.33,
//     src/linear_algebra.zig:67): for n == 2 the tridiagonal reduction is the
//     identity and dsteqr finishes with dlaev2 + one plane rotation; n >= 3
//     runs dsytd2, dsteqr (implicit QL/QR, dlartg of LAPACK >= 3.10) and
//     dorm2l.  The eigenvector signs are LAPACK's (pinned against
//     numpy.linalg.eigh(UPLO='U'), which calls LAPACK dsyevd, in the tests).
//   * custom potentials: an own recursive-descent evaluator of the ExprTk
//     subset used by Zinq inputs (src/exprtk.cpp:10-40).
//
// Build: oracle/Makefile (g++ -O3 -ffp-contract=off -fopenmp -shared).

#include "qd_ref.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

struct cplx {
    double re, im;
};
inline cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
inline cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
// std.math.Complex.mul
inline cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cplx cconj(cplx a) { return {a.re, -a.im}; }
// std.math.Complex.div
inline cplx cdiv(cplx a, cplx b) {
    double re_num = a.re * b.re + a.im * b.im;
    double im_num = a.im * b.re - a.re * b.im;
    double den = b.re * b.re + b.im * b.im;
    return {re_num / den, im_num / den};
}
// std.math.complex.exp (musl cexp special cases give identical values)
inline cplx cexp_(cplx z) {
    if (z.im == 0.0) return {std::exp(z.re), z.im};
    if (z.re == 0.0) return {std::cos(z.im), std::sin(z.im)};
    double e = std::exp(z.re);
    return {e * std::cos(z.im), e * std::sin(z.im)};
}
inline double sqmag(cplx a) { return a.re * a.re + a.im * a.im; }

// ---------------------------------------------------------------- expressions
// Subset of ExprTk (src/exprtk.cpp:10-26: variables r1..rN and t plus the
// constants pi, epsilon, inf).  Precedence: comparison < +,- < *,/,% <
// unary sign < ^ (left-associative).  Constant integer exponents are
// evaluated by binary powering, others by pow().
struct Node {
    enum K { NUM, VAR, TIME, NEG, ADD, SUB, MUL, DIV, MOD, POW, IPOW, LT, LE, GT, GE, EQ, NE, FN1, FN2, FNV, IF } k;
    double v = 0;
    int idx = 0;
    std::string fn;
    std::vector<std::unique_ptr<Node>> c;
};

struct Parser {
    const std::string& s;
    size_t p = 0;
    int nvar;
    explicit Parser(const std::string& str, int nv) : s(str), nvar(nv) {}
    void ws() {
        while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
    }
    bool eat(const char* tok) {
        ws();
        size_t L = std::strlen(tok);
        if (s.compare(p, L, tok) == 0) {
            p += L;
            return true;
        }
        return false;
    }
    [[noreturn]] void fail(const std::string& m) { throw std::runtime_error(m + " at offset " + std::to_string(p)); }
    static std::unique_ptr<Node> mk(Node::K k) {
        auto n = std::make_unique<Node>();
        n->k = k;
        return n;
    }
    static std::unique_ptr<Node> bin(Node::K k, std::unique_ptr<Node> a, std::unique_ptr<Node> b) {
        auto n = mk(k);
        n->c.push_back(std::move(a));
        n->c.push_back(std::move(b));
        return n;
    }
    std::unique_ptr<Node> parse() {
        auto e = expr();
        ws();
        if (p != s.size()) fail("unexpected trailing input");
        return e;
    }
    std::unique_ptr<Node> expr() {
        auto a = additive();
        for (;;) {
            ws();
            Node::K k;
            if (eat("<=")) k = Node::LE;
            else if (eat(">=")) k = Node::GE;
            else if (eat("==")) k = Node::EQ;
            else if (eat("!=") || eat("<>")) k = Node::NE;
            else if (eat("<")) k = Node::LT;
            else if (eat(">")) k = Node::GT;
            else if (eat("=")) k = Node::EQ;
            else return a;
            a = bin(k, std::move(a), additive());
        }
    }
    std::unique_ptr<Node> additive() {
        auto a = term();
        for (;;) {
            if (eat("+")) a = bin(Node::ADD, std::move(a), term());
            else if (eat("-")) a = bin(Node::SUB, std::move(a), term());
            else return a;
        }
    }
    std::unique_ptr<Node> term() {
        auto a = unary();
        for (;;) {
            if (eat("*")) a = bin(Node::MUL, std::move(a), unary());
            else if (eat("/")) a = bin(Node::DIV, std::move(a), unary());
            else if (eat("%")) a = bin(Node::MOD, std::move(a), unary());
            else {
                // implicit multiplication: "2x", "2(x+1)", ")(" like ExprTk
                ws();
                if (p < s.size() && (std::isalpha((unsigned char)s[p]) || s[p] == '(') && prev_implicit_ok) {
                    prev_implicit_ok = false;
                    a = bin(Node::MUL, std::move(a), unary());
                } else
                    return a;
            }
        }
    }
    bool prev_implicit_ok = false;
    std::unique_ptr<Node> unary() {
        if (eat("-")) {
            auto n = mk(Node::NEG);
            n->c.push_back(unary());
            return n;
        }
        if (eat("+")) return unary();
        return power();
    }
    std::unique_ptr<Node> signed_primary() {
        if (eat("-")) {
            auto n = mk(Node::NEG);
            n->c.push_back(signed_primary());
            return n;
        }
        if (eat("+")) return signed_primary();
        return primary();
    }
    std::unique_ptr<Node> power() {
        auto a = primary();
        while (eat("^")) {
            auto b = signed_primary();
            a = make_pow(std::move(a), std::move(b));
        }
        return a;
    }
    static std::unique_ptr<Node> make_pow(std::unique_ptr<Node> a, std::unique_ptr<Node> b) {
        const Node* e = b.get();
        double sign = 1;
        while (e->k == Node::NEG) {
            sign = -sign;
            e = e->c[0].get();
        }
        if (e->k == Node::NUM) {
            double v = sign * e->v;
            if (v == std::floor(v) && std::fabs(v) <= 64) {
                auto n = mk(Node::IPOW);
                n->idx = (int)v;
                n->c.push_back(std::move(a));
                return n;
            }
        }
        return bin(Node::POW, std::move(a), std::move(b));
    }
    std::unique_ptr<Node> primary() {
        ws();
        prev_implicit_ok = false;
        if (p >= s.size()) fail("unexpected end of expression");
        char ch = s[p];
        if (ch == '(') {
            ++p;
            auto e = expr();
            if (!eat(")")) fail("expected ')'");
            prev_implicit_ok = true;
            return e;
        }
        if (std::isdigit((unsigned char)ch) || ch == '.') {
            size_t q = p;
            while (q < s.size() && (std::isdigit((unsigned char)s[q]) || s[q] == '.')) ++q;
            if (q < s.size() && (s[q] == 'e' || s[q] == 'E')) {
                size_t r = q + 1;
                if (r < s.size() && (s[r] == '+' || s[r] == '-')) ++r;
                if (r < s.size() && std::isdigit((unsigned char)s[r])) {
                    q = r;
                    while (q < s.size() && std::isdigit((unsigned char)s[q])) ++q;
                }
            }
            std::string num = s.substr(p, q - p);
            char* endp = nullptr;
            double v = std::strtod(num.c_str(), &endp);
            if (!endp || *endp != '\0') fail("bad number");
            p = q;
            auto n = mk(Node::NUM);
            n->v = v;
            prev_implicit_ok = true;
            return n;
        }
        if (std::isalpha((unsigned char)ch) || ch == '_') {
            size_t q = p;
            while (q < s.size() && (std::isalnum((unsigned char)s[q]) || s[q] == '_')) ++q;
            std::string id = s.substr(p, q - p);
            p = q;
            std::string lid = id;
            for (auto& c : lid) c = (char)std::tolower((unsigned char)c);
            ws();
            if (p < s.size() && s[p] == '(') {
                ++p;
                std::vector<std::unique_ptr<Node>> args;
                ws();
                if (!eat(")")) {
                    for (;;) {
                        args.push_back(expr());
                        if (eat(",")) continue;
                        if (eat(")")) break;
                        fail("expected ',' or ')'");
                    }
                }
                static const char* f1[] = {"abs", "sgn", "exp", "log", "log10", "log2", "sqrt", "sin", "cos", "tan",
                                           "asin", "acos", "atan", "sinh", "cosh", "tanh", "erf", "erfc", "floor",
                                           "ceil", "round", "trunc", "log1p", "expm1", "cbrt"};
                static const char* f2[] = {"pow", "atan2", "hypot", "fmod"};
                for (auto f : f1)
                    if (lid == f) {
                        if (args.size() != 1) fail("function " + id + " takes 1 argument");
                        auto n = mk(Node::FN1);
                        n->fn = lid;
                        n->c = std::move(args);
                        prev_implicit_ok = true;
                        return n;
                    }
                for (auto f : f2)
                    if (lid == f) {
                        if (args.size() != 2) fail("function " + id + " takes 2 arguments");
                        if (lid == "pow") {
                            auto a0 = std::move(args[0]);
                            auto a1 = std::move(args[1]);
                            prev_implicit_ok = true;
                            return make_pow(std::move(a0), std::move(a1));
                        }
                        auto n = mk(Node::FN2);
                        n->fn = lid;
                        n->c = std::move(args);
                        prev_implicit_ok = true;
                        return n;
                    }
                if (lid == "min" || lid == "max") {
                    if (args.empty()) fail(id + " needs arguments");
                    auto n = mk(Node::FNV);
                    n->fn = lid;
                    n->c = std::move(args);
                    prev_implicit_ok = true;
                    return n;
                }
                if (lid == "if") {
                    if (args.size() != 3) fail("if takes 3 arguments");
                    auto n = mk(Node::IF);
                    n->c = std::move(args);
                    prev_implicit_ok = true;
                    return n;
                }
                fail("unknown function " + id);
            }
            prev_implicit_ok = true;
            if (lid == "pi") {
                auto n = mk(Node::NUM);
                n->v = 3.141592653589793238462643383279502;
                return n;
            }
            if (lid == "epsilon") {
                auto n = mk(Node::NUM);
                n->v = std::numeric_limits<double>::epsilon();
                return n;
            }
            if (lid == "inf") {
                auto n = mk(Node::NUM);
                n->v = std::numeric_limits<double>::infinity();
                return n;
            }
            if (id == "t") return mk(Node::TIME);
            if (id.size() >= 2 && id[0] == 'r') {
                bool digits = true;
                for (size_t i = 1; i < id.size(); ++i) digits = digits && std::isdigit((unsigned char)id[i]);
                if (digits) {
                    int k = std::atoi(id.c_str() + 1);
                    if (k >= 1 && k <= nvar) {
                        auto n = mk(Node::VAR);
                        n->idx = k - 1;
                        return n;
                    }
                }
            }
            fail("unknown symbol " + id);
        }
        fail(std::string("unexpected character '") + ch + "'");
    }
};

double ipow(double x, int e) {
    bool neg = e < 0;
    unsigned u = (unsigned)(neg ? -e : e);
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
    return neg ? 1.0 / result : result;
}

double eval(const Node* n, const double* r, double t) {
    switch (n->k) {
    case Node::NUM: return n->v;
    case Node::VAR: return r[n->idx];
    case Node::TIME: return t;
    case Node::NEG: return -eval(n->c[0].get(), r, t);
    case Node::ADD: return eval(n->c[0].get(), r, t) + eval(n->c[1].get(), r, t);
    case Node::SUB: return eval(n->c[0].get(), r, t) - eval(n->c[1].get(), r, t);
    case Node::MUL: return eval(n->c[0].get(), r, t) * eval(n->c[1].get(), r, t);
    case Node::DIV: return eval(n->c[0].get(), r, t) / eval(n->c[1].get(), r, t);
    case Node::MOD: return std::fmod(eval(n->c[0].get(), r, t), eval(n->c[1].get(), r, t));
    case Node::POW: return std::pow(eval(n->c[0].get(), r, t), eval(n->c[1].get(), r, t));
    case Node::IPOW: return ipow(eval(n->c[0].get(), r, t), n->idx);
    case Node::LT: return eval(n->c[0].get(), r, t) < eval(n->c[1].get(), r, t) ? 1.0 : 0.0;
    case Node::LE: return eval(n->c[0].get(), r, t) <= eval(n->c[1].get(), r, t) ? 1.0 : 0.0;
    case Node::GT: return eval(n->c[0].get(), r, t) > eval(n->c[1].get(), r, t) ? 1.0 : 0.0;
    case Node::GE: return eval(n->c[0].get(), r, t) >= eval(n->c[1].get(), r, t) ? 1.0 : 0.0;
    case Node::EQ: return eval(n->c[0].get(), r, t) == eval(n->c[1].get(), r, t) ? 1.0 : 0.0;
    case Node::NE: return eval(n->c[0].get(), r, t) != eval(n->c[1].get(), r, t) ? 1.0 : 0.0;
    case Node::IF: return eval(n->c[0].get(), r, t) != 0.0 ? eval(n->c[1].get(), r, t) : eval(n->c[2].get(), r, t);
    case Node::FNV: {
        double v = eval(n->c[0].get(), r, t);
        for (size_t i = 1; i < n->c.size(); ++i) {
            double w = eval(n->c[i].get(), r, t);
            v = n->fn == "min" ? (w < v ? w : v) : (w > v ? w : v);
        }
        return v;
    }
    case Node::FN2: {
        double a = eval(n->c[0].get(), r, t), b = eval(n->c[1].get(), r, t);
        if (n->fn == "atan2") return std::atan2(a, b);
        if (n->fn == "hypot") return std::hypot(a, b);
        return std::fmod(a, b);
    }
    case Node::FN1: {
        double x = eval(n->c[0].get(), r, t);
        const std::string& f = n->fn;
        if (f == "abs") return std::fabs(x);
        if (f == "sgn") return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0);
        if (f == "exp") return std::exp(x);
        if (f == "log") return std::log(x);
        if (f == "log10") return std::log10(x);
        if (f == "log2") return std::log2(x);
        if (f == "sqrt") return std::sqrt(x);
        if (f == "sin") return std::sin(x);
        if (f == "cos") return std::cos(x);
        if (f == "tan") return std::tan(x);
        if (f == "asin") return std::asin(x);
        if (f == "acos") return std::acos(x);
        if (f == "atan") return std::atan(x);
        if (f == "sinh") return std::sinh(x);
        if (f == "cosh") return std::cosh(x);
        if (f == "tanh") return std::tanh(x);
        if (f == "erf") return std::erf(x);
        if (f == "erfc") return std::erfc(x);
        if (f == "floor") return std::floor(x);
        if (f == "ceil") return std::ceil(x);
        if (f == "round") return std::round(x);
        if (f == "trunc") return std::trunc(x);
        if (f == "log1p") return std::log1p(x);
        if (f == "expm1") return std::expm1(x);
        if (f == "cbrt") return std::cbrt(x);
        return NAN;
    }
    }
    return NAN;
}

std::unique_ptr<Node> compile_expr(const std::string& s, int nvar) {
    Parser ps(s, nvar);
    return ps.parse();
}

// ----------------------------------------------------------------------- FFT
// One 1-D transform length with precomputed twiddles.
struct Fft1 {
    size_t n = 0;
    bool pow2 = true;
    std::vector<uint32_t> rev;
    std::vector<cplx> tw; // exp(-2 pi i k / n), k < n/2 (power of two)
    // Bluestein for non-power-of-two n
    size_t m = 0;
    std::vector<cplx> chirp;  // exp(-pi i k^2 / n)
    std::vector<cplx> filt_f; // FFT_m of conj chirp (forward)
    std::unique_ptr<Fft1> sub;

    static cplx unit(long double frac) { // exp(-2 pi i frac), frac in [0,1)
        const long double tau = 6.283185307179586476925286766559005768L;
        long double a = tau * frac;
        return {(double)cosl(a), (double)-sinl(a)};
    }
    explicit Fft1(size_t len) : n(len) {
        pow2 = (n & (n - 1)) == 0;
        if (pow2) {
            int lg = 0;
            while ((size_t(1) << lg) < n) ++lg;
            rev.resize(n);
            for (size_t i = 0; i < n; ++i) {
                uint32_t r = 0;
                for (int b = 0; b < lg; ++b)
                    if (i & (size_t(1) << b)) r |= 1u << (lg - 1 - b);
                rev[i] = r;
            }
            tw.resize(n / 2 > 0 ? n / 2 : 1);
            for (size_t k = 0; k < n / 2; ++k) tw[k] = unit((long double)k / (long double)n);
        } else {
            m = 1;
            while (m < 2 * n - 1) m <<= 1;
            sub = std::make_unique<Fft1>(m);
            chirp.resize(n);
            for (size_t k = 0; k < n; ++k) {
                unsigned long long kk = (unsigned long long)k * k % (2ull * n);
                chirp[k] = unit((long double)kk / (long double)(2 * n));
            }
            filt_f.assign(m, {0, 0});
            filt_f[0] = cconj(chirp[0]);
            for (size_t k = 1; k < n; ++k) filt_f[k] = filt_f[m - k] = cconj(chirp[k]);
            sub->run(filt_f.data(), -1);
        }
    }
    // unnormalised transform of x (contiguous), sign -1 or +1
    void run(cplx* x, int sign) const {
        if (n <= 1) return;
        if (pow2) {
            for (size_t i = 0; i < n; ++i)
                if (rev[i] > i) std::swap(x[i], x[rev[i]]);
            for (size_t len = 2; len <= n; len <<= 1) {
                size_t half = len / 2, step = n / len;
                for (size_t i = 0; i < n; i += len)
                    for (size_t j = 0; j < half; ++j) {
                        cplx w = tw[j * step];
                        if (sign > 0) w.im = -w.im;
                        cplx u = x[i + j], v = cmul(x[i + j + half], w);
                        x[i + j] = cadd(u, v);
                        x[i + j + half] = csub(u, v);
                    }
            }
            return;
        }
        std::vector<cplx> a(m, {0, 0});
        for (size_t k = 0; k < n; ++k) {
            cplx c = sign < 0 ? chirp[k] : cconj(chirp[k]);
            a[k] = cmul(x[k], c);
        }
        sub->run(a.data(), -1);
        if (sign < 0) {
            for (size_t k = 0; k < m; ++k) a[k] = cmul(a[k], filt_f[k]);
        } else {
            // filter with chirp instead of its conjugate: FFT(conj(h)) = conj(FFT(h) reversed)
            for (size_t k = 0; k < m; ++k) a[k] = cmul(a[k], cconj(filt_f[(m - k) % m]));
        }
        sub->run(a.data(), +1);
        double inv = 1.0 / (double)m;
        for (size_t k = 0; k < n; ++k) {
            cplx c = sign < 0 ? chirp[k] : cconj(chirp[k]);
            cplx v = {a[k].re * inv, a[k].im * inv};
            x[k] = cmul(v, c);
        }
    }
};

// N-D in-place transform over a row-major n^d array (fftw_plan_dft,
// src/fourier_transform.zig:15-23; execute + 1/N loop :38-47).
struct FftNd {
    int d;
    size_t n, N;
    std::unique_ptr<Fft1> f;
    FftNd(int ndim, size_t npt) : d(ndim), n(npt) {
        N = 1;
        for (int i = 0; i < d; ++i) N *= n;
        f = std::make_unique<Fft1>(n);
    }
    void execute(cplx* x, int sign, int nthreads) const {
        for (int a = d - 1; a >= 0; --a) {
            size_t stride = 1;
            for (int b = a + 1; b < d; ++b) stride *= n;
            size_t nlines = N / n;
#pragma omp parallel for num_threads(nthreads) if (nthreads > 1 && nlines > 1) schedule(static)
            for (size_t l = 0; l < nlines; ++l) {
                size_t outer = l / stride, inner = l % stride;
                size_t base = outer * stride * n + inner;
                if (stride == 1) {
                    f->run(x + base, sign);
                } else {
                    std::vector<cplx> buf(n);
                    for (size_t i = 0; i < n; ++i) buf[i] = x[base + i * stride];
                    f->run(buf.data(), sign);
                    for (size_t i = 0; i < n; ++i) x[base + i * stride] = buf[i];
                }
            }
        }
        if (sign == 1) {
            double dn = (double)N;
            for (size_t i = 0; i < N; ++i) {
                x[i].re /= dn;
                x[i].im /= dn;
            }
        }
    }
};

// --------------------------------------------------------------------- eigh
// dlaev2: eigensystem of [[a,b],[b,c]] (LAPACK, published algorithm).
void dlaev2(double a, double b, double c, double& rt1, double& rt2, double& cs1, double& sn1) {
    double sm = a + c, df = a - c, adf = std::fabs(df), tb = b + b, ab = std::fabs(tb);
    double acmx, acmn, rt, cs, ct, tn;
    int sgn1, sgn2;
    if (std::fabs(a) > std::fabs(c)) {
        acmx = a;
        acmn = c;
    } else {
        acmx = c;
        acmn = a;
    }
    if (adf > ab) rt = adf * std::sqrt(1.0 + (ab / adf) * (ab / adf));
    else if (adf < ab) rt = ab * std::sqrt(1.0 + (adf / ab) * (adf / ab));
    else rt = ab * std::sqrt(2.0);
    if (sm < 0.0) {
        rt1 = 0.5 * (sm - rt);
        sgn1 = -1;
        rt2 = (acmx / rt1) * acmn - (b / rt1) * b;
    } else if (sm > 0.0) {
        rt1 = 0.5 * (sm + rt);
        sgn1 = 1;
        rt2 = (acmx / rt1) * acmn - (b / rt1) * b;
    } else {
        rt1 = 0.5 * rt;
        rt2 = -0.5 * rt;
        sgn1 = 1;
    }
    if (df >= 0.0) {
        cs = df + rt;
        sgn2 = 1;
    } else {
        cs = df - rt;
        sgn2 = -1;
    }
    double acs = std::fabs(cs);
    if (acs > ab) {
        ct = -tb / cs;
        sn1 = 1.0 / std::sqrt(1.0 + ct * ct);
        cs1 = ct * sn1;
    } else {
        if (ab == 0.0) {
            cs1 = 1.0;
            sn1 = 0.0;
        } else {
            tn = -cs / tb;
            cs1 = 1.0 / std::sqrt(1.0 + tn * tn);
            sn1 = tn * cs1;
        }
    }
    if (sgn1 == sgn2) {
        tn = cs1;
        cs1 = -sn1;
        sn1 = tn;
    }
}

// dsyevd for a 2x2 symmetric matrix: dsytrd is the identity, dstedc -> dsteqr.
void eigh2(const double* V, double* W, double* U) {
    const double eps = std::ldexp(1.0, -53), eps2 = eps * eps, safmin = std::numeric_limits<double>::min();
    double d1 = V[0], d2 = V[3], e = V[1];
    double z11 = 1, z12 = 0, z21 = 0, z22 = 1;
    bool rotate = false;
    double tst = std::fabs(e);
    bool split = (tst == 0.0) || (tst <= (std::sqrt(std::fabs(d1)) * std::sqrt(std::fabs(d2))) * eps);
    if (!split) {
        double anorm = std::max(std::max(std::fabs(d1), std::fabs(d2)), std::fabs(e));
        if (anorm != 0.0) {
            if (std::fabs(d2) < std::fabs(d1)) { // QR branch, L=2, LEND=1
                double t2 = std::fabs(e) * std::fabs(e);
                rotate = !(t2 <= (eps2 * std::fabs(d2)) * std::fabs(d1) + safmin);
            } else { // QL branch, L=1, LEND=2
                double t2 = std::fabs(e) * std::fabs(e);
                rotate = !(t2 <= (eps2 * std::fabs(d1)) * std::fabs(d2) + safmin);
            }
        }
    }
    if (rotate) {
        double rt1, rt2, c, s;
        dlaev2(d1, e, d2, rt1, rt2, c, s);
        // dlasr('R','V',*) on the identity: Z = [[c,-s],[s,c]]
        z11 = c;
        z21 = s;
        z12 = -s;
        z22 = c;
        d1 = rt1;
        d2 = rt2;
    }
    if (d2 < d1) { // selection sort with column swap
        std::swap(d1, d2);
        std::swap(z11, z12);
        std::swap(z21, z22);
    }
    W[0] = d1;
    W[1] = d2;
    U[0] = z11;
    U[1] = z12;
    U[2] = z21;
    U[3] = z22;
}

// LAPACK dsyevd('V', 'U') for small n (the reference's eighBatch, src/linear_algebra.zig:55-70,
// calls LAPACKE_dsyevd row-major; for symmetric input that is dsyevd on the same matrix), restated
// from the published netlib algorithm: dsytd2 (Householder reduction of the upper triangle, last
// column first), dsteqr('I') (implicit QL or QR with Wilkinson-type shifts and plane rotations,
// 2 x 2 blocks by dlaev2, selection sort of the eigenvalues) and dorm2l (the reflectors applied
// to the eigenvectors of the tridiagonal matrix).  Arithmetic in the published operation order.
namespace lapack {
const double EPS = 1.1102230246251565e-16;    // dlamch('E') = 2^-53
const double SAFMIN = 2.2250738585072014e-308; // dlamch('S')

double sign(double a, double b) { return b >= 0 ? std::fabs(a) : -std::fabs(a); }

double dlapy2(double x, double y) {
    const double xa = std::fabs(x), ya = std::fabs(y), w = std::max(xa, ya), z = std::min(xa, ya);
    if (z == 0.0 || w > 1.7976931348623157e308) return w;
    const double q = z / w;
    return w * std::sqrt(1.0 + q * q);
}

// dlartg (LAPACK >= 3.10): c >= 0, r carries the sign of f
void dlartg(double f, double g, double& c, double& s, double& r) {
    const double rtmin = std::sqrt(SAFMIN), rtmax = std::sqrt(1.0 / SAFMIN / 2.0);
    const double f1 = std::fabs(f), g1 = std::fabs(g);
    if (g == 0.0) {
        c = 1.0;
        s = 0.0;
        r = f;
    } else if (f == 0.0) {
        c = 0.0;
        s = sign(1.0, g);
        r = g1;
    } else if (f1 > rtmin && f1 < rtmax && g1 > rtmin && g1 < rtmax) {
        const double d = std::sqrt(f * f + g * g);
        c = f1 / d;
        r = sign(d, f);
        s = g / r;
    } else {
        const double u = std::min(1.0 / SAFMIN, std::max(SAFMIN, std::max(f1, g1)));
        const double fs = f / u, gs = g / u, d = std::sqrt(fs * fs + gs * gs);
        c = std::fabs(fs) / d;
        r = sign(d, f);
        s = gs / r;
        r = r * u;
    }
}

// dlasr('R', 'V', DIRECT, m rows, cols j0 .. j0+nc-1 of Z (n x n, column j of Z at Z[r*n + j]))
void dlasr_rv(bool forward, int n, int j0, int nc, const double* c, const double* s, double* Z) {
    auto rot = [&](int j) {
        const double ct = c[j], st = s[j];
        if (ct == 1.0 && st == 0.0) return;
        for (int i = 0; i < n; ++i) {
            const double t = Z[i * n + j0 + j + 1];
            Z[i * n + j0 + j + 1] = ct * t - st * Z[i * n + j0 + j];
            Z[i * n + j0 + j] = st * t + ct * Z[i * n + j0 + j];
        }
    };
    if (forward)
        for (int j = 0; j < nc - 1; ++j) rot(j);
    else
        for (int j = nc - 2; j >= 0; --j) rot(j);
}

// dsteqr('I'): eigenvalues d (ascending on return) and eigenvectors Z of the tridiagonal (d, e)
bool dsteqr(int n, double* d, double* e, double* Z) {
    const double eps2 = EPS * EPS, safmax = 1.0 / SAFMIN, ssfmax = std::sqrt(safmax) / 3.0,
                 ssfmin = std::sqrt(SAFMIN) / eps2;
    for (int i = 0; i < n * n; ++i) Z[i] = 0.0;
    for (int i = 0; i < n; ++i) Z[i * n + i] = 1.0;
    double wc[8], ws[8]; // work(1:n-1) and work(n:2n-2)
    const int nmaxit = n * 30;
    int jtot = 0, l1 = 0;
    for (;;) { // 10
        if (l1 > n - 1) break;
        if (l1 > 0) e[l1 - 1] = 0.0;
        int m = n - 1;
        for (int mm = l1; mm < n - 1; ++mm) {
            const double tst = std::fabs(e[mm]);
            if (tst == 0.0) {
                m = mm;
                break;
            }
            if (tst <= (std::sqrt(std::fabs(d[mm])) * std::sqrt(std::fabs(d[mm + 1]))) * EPS) {
                e[mm] = 0.0;
                m = mm;
                break;
            }
        }
        int l = l1;
        const int lsv = l;
        int lend = m;
        const int lendsv = lend;
        l1 = m + 1;
        if (lend == l) continue;
        // scale the block (only outside [ssfmin, ssfmax])
        double anorm = 0.0;
        for (int i = l; i <= lend; ++i) anorm = std::max(anorm, std::fabs(d[i]));
        for (int i = l; i < lend; ++i) anorm = std::max(anorm, std::fabs(e[i]));
        if (anorm == 0.0) continue;
        double to = 0.0; // dlascl: the block scaled by to / anorm (outside [ssfmin, ssfmax] only)
        if (anorm > ssfmax) to = ssfmax;
        if (anorm < ssfmin) to = ssfmin;
        if (to != 0.0) {
            for (int i = l; i <= lend; ++i) d[i] = d[i] * (to / anorm);
            for (int i = l; i < lend; ++i) e[i] = e[i] * (to / anorm);
        }
        if (std::fabs(d[lend]) < std::fabs(d[l])) {
            lend = lsv;
            l = lendsv;
        }
        if (lend > l) { // QL iteration
            for (;;) {   // 40
                int mq = lend;
                for (int mm = l; mm < lend; ++mm) {
                    const double tst = std::fabs(e[mm]) * std::fabs(e[mm]);
                    if (tst <= (eps2 * std::fabs(d[mm])) * std::fabs(d[mm + 1]) + SAFMIN) {
                        mq = mm;
                        break;
                    }
                }
                if (mq < lend) e[mq] = 0.0;
                double p = d[l];
                if (mq == l) { // eigenvalue found
                    d[l] = p;
                    ++l;
                    if (l <= lend) continue;
                    break;
                }
                if (mq == l + 1) {
                    double rt1, rt2, c, s;
                    dlaev2(d[l], e[l], d[l + 1], rt1, rt2, c, s);
                    wc[0] = c;
                    ws[0] = s;
                    dlasr_rv(false, n, l, 2, wc, ws, Z);
                    d[l] = rt1;
                    d[l + 1] = rt2;
                    e[l] = 0.0;
                    l += 2;
                    if (l <= lend) continue;
                    break;
                }
                if (jtot == nmaxit) break;
                ++jtot;
                double g = (d[l + 1] - p) / (2.0 * e[l]);
                double r = dlapy2(g, 1.0);
                g = d[mq] - p + (e[l] / (g + sign(r, g)));
                double s = 1.0, c = 1.0;
                p = 0.0;
                for (int i = mq - 1; i >= l; --i) {
                    const double f = s * e[i], b = c * e[i];
                    dlartg(g, f, c, s, r);
                    if (i != mq - 1) e[i + 1] = r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    p = s * r;
                    d[i + 1] = g + p;
                    g = c * r - b;
                    wc[i - l] = c;
                    ws[i - l] = -s;
                }
                dlasr_rv(false, n, l, mq - l + 1, wc, ws, Z);
                d[l] = d[l] - p;
                e[l] = g;
            }
        } else { // QR iteration
            for (;;) { // 90
                int mq = lend;
                for (int mm = l; mm > lend; --mm) {
                    const double tst = std::fabs(e[mm - 1]) * std::fabs(e[mm - 1]);
                    if (tst <= (eps2 * std::fabs(d[mm])) * std::fabs(d[mm - 1]) + SAFMIN) {
                        mq = mm;
                        break;
                    }
                }
                if (mq > lend) e[mq - 1] = 0.0;
                double p = d[l];
                if (mq == l) {
                    d[l] = p;
                    --l;
                    if (l >= lend) continue;
                    break;
                }
                if (mq == l - 1) {
                    double rt1, rt2, c, s;
                    dlaev2(d[l - 1], e[l - 1], d[l], rt1, rt2, c, s);
                    wc[0] = c;
                    ws[0] = s;
                    dlasr_rv(true, n, l - 1, 2, wc, ws, Z);
                    d[l - 1] = rt1;
                    d[l] = rt2;
                    e[l - 1] = 0.0;
                    l -= 2;
                    if (l >= lend) continue;
                    break;
                }
                if (jtot == nmaxit) break;
                ++jtot;
                double g = (d[l - 1] - p) / (2.0 * e[l - 1]);
                double r = dlapy2(g, 1.0);
                g = d[mq] - p + (e[l - 1] / (g + sign(r, g)));
                double s = 1.0, c = 1.0;
                p = 0.0;
                for (int i = mq; i <= l - 1; ++i) {
                    const double f = s * e[i], b = c * e[i];
                    dlartg(g, f, c, s, r);
                    if (i != mq) e[i - 1] = r;
                    g = d[i] - p;
                    r = (d[i + 1] - g) * s + 2.0 * c * b;
                    p = s * r;
                    d[i] = g + p;
                    g = c * r - b;
                    wc[i - mq] = c;
                    ws[i - mq] = s;
                }
                dlasr_rv(true, n, mq, l - mq + 1, wc, ws, Z);
                d[l] = d[l] - p;
                e[l - 1] = g;
            }
        }
        if (to != 0.0) { // undo the scaling
            for (int i = lsv; i <= lendsv; ++i) d[i] = d[i] * (anorm / to);
            for (int i = lsv; i < lendsv; ++i) e[i] = e[i] * (anorm / to);
        }
        if (jtot >= nmaxit) return false;
    }
    for (int ii = 1; ii < n; ++ii) { // selection sort, ascending
        const int i = ii - 1;
        int k = i;
        double p = d[i];
        for (int j = ii; j < n; ++j)
            if (d[j] < p) {
                k = j;
                p = d[j];
            }
        if (k != i) {
            d[k] = d[i];
            d[i] = p;
            for (int r = 0; r < n; ++r) std::swap(Z[r * n + i], Z[r * n + k]);
        }
    }
    return true;
}

// dsyevd('V', 'U') of the symmetric n x n V (row-major; the upper triangle is read)
void dsyevd(int n, const double* V, double* W, double* U) {
    double A[8][8] = {}, d[8] = {}, e[8] = {}, tau[8] = {}; // A[i][j]: LAPACK's A(i+1, j+1)
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) A[i][j] = V[i * n + j];
    // dsytd2('U'): reflector H(i) annihilates A(1:i-1, i+1), i = n-1 .. 1
    for (int i = n - 1; i >= 1; --i) {
        // dlarfg(i, A(i, i+1), A(1:i-1, i+1))
        double alpha = A[i - 1][i], taui = 0.0;
        if (i > 1) {
            // dnrm2 of A(1:i-1, i+1), scaled by the largest magnitude so that tiny couplings do not
            // underflow (a naive sum of squares of 1e-162 is denormal and breaks the reflector)
            double big = 0.0;
            for (int k = 0; k < i - 1; ++k) big = std::max(big, std::fabs(A[k][i]));
            double xnorm = 0.0;
            if (big > 0.0) {
                double ssq = 0.0;
                for (int k = 0; k < i - 1; ++k) {
                    const double q = A[k][i] / big;
                    ssq += q * q;
                }
                xnorm = big * std::sqrt(ssq);
            }
            if (xnorm != 0.0) {
                double beta = -sign(dlapy2(alpha, xnorm), alpha);
                // dlarfg's rescaling: while |beta| < safmin / eps, scale x and alpha by eps / safmin
                const double sfmin = SAFMIN / EPS, rsafmn = 1.0 / sfmin;
                int knt = 0;
                if (std::fabs(beta) < sfmin) {
                    do {
                        ++knt;
                        for (int k = 0; k < i - 1; ++k) A[k][i] = A[k][i] * rsafmn;
                        beta = beta * rsafmn;
                        alpha = alpha * rsafmn;
                    } while (std::fabs(beta) < sfmin && knt < 20);
                    double big2 = 0.0, ssq = 0.0;
                    for (int k = 0; k < i - 1; ++k) big2 = std::max(big2, std::fabs(A[k][i]));
                    for (int k = 0; k < i - 1; ++k) {
                        const double q = A[k][i] / big2;
                        ssq += q * q;
                    }
                    beta = -sign(dlapy2(alpha, big2 * std::sqrt(ssq)), alpha);
                }
                taui = (beta - alpha) / beta;
                const double sc = 1.0 / (alpha - beta);
                for (int k = 0; k < i - 1; ++k) A[k][i] = A[k][i] * sc;
                for (int j = 0; j < knt; ++j) beta = beta * sfmin;
                alpha = beta;
            }
        }
        A[i - 1][i] = alpha;
        e[i - 1] = alpha;
        if (taui != 0.0) {
            A[i - 1][i] = 1.0;
            // tau(1:i) = taui * A(1:i, 1:i) v, v = A(1:i, i+1) (dsymv, upper)
            double y[8] = {0};
            for (int j = 0; j < i; ++j) {
                const double t1 = taui * A[j][i];
                double t2 = 0.0;
                for (int k = 0; k < j; ++k) {
                    y[k] += t1 * A[k][j];
                    t2 += A[k][j] * A[k][i];
                }
                y[j] += t1 * A[j][j] + taui * t2;
            }
            double dot = 0.0;
            for (int k = 0; k < i; ++k) dot += y[k] * A[k][i];
            const double al = -0.5 * taui * dot;
            for (int k = 0; k < i; ++k) y[k] += al * A[k][i];
            // A := A - v w' - w v' (dsyr2, upper)
            for (int j = 0; j < i; ++j) {
                if (A[j][i] != 0.0 || y[j] != 0.0) {
                    const double t1 = -1.0 * y[j], t2 = -1.0 * A[j][i];
                    for (int k = 0; k <= j; ++k) A[k][j] += A[k][i] * t1 + y[k] * t2;
                }
            }
            A[i - 1][i] = e[i - 1];
        }
        d[i] = A[i][i];
        tau[i - 1] = taui;
    }
    d[0] = A[0][0];
    double Z[64];
    if (!dsteqr(n, d, e, Z)) throw std::runtime_error("dsteqr did not converge");
    // dorm2l('L', 'N'): Z(1:i, :) <- H(i) Z(1:i, :), i = 1 .. n-1, v = [A(1:i-1, i+1); 1]
    for (int i = 1; i <= n - 1; ++i) {
        const double t = tau[i - 1];
        if (t == 0.0) continue;
        double v[8];
        for (int k = 0; k < i - 1; ++k) v[k] = A[k][i];
        v[i - 1] = 1.0;
        for (int c = 0; c < n; ++c) {
            double w = 0.0;
            for (int k = 0; k < i; ++k) w += Z[k * n + c] * v[k];
            for (int k = 0; k < i; ++k) Z[k * n + c] -= t * v[k] * w;
        }
    }
    for (int i = 0; i < n; ++i) W[i] = d[i];
    for (int i = 0; i < n * n; ++i) U[i] = Z[i];
}
} // namespace lapack

void eigh_any(int n, const double* V, double* W, double* U) {
    if (n == 1) {
        W[0] = V[0];
        U[0] = 1.0;
    } else if (n == 2) {
        eigh2(V, W, U);
    } else {
        lapack::dsyevd(n, V, W, U);
    }
}

// ---------------------------------------------------------------- potential
// src/potential.zig:63-615
struct Potential {
    int kind;
    int nd = 1, ns = 1;
    bool td = false;
    std::vector<double> prm;
    std::vector<std::unique_ptr<Node>> ex;
    std::vector<double> freq, exc, kap, lmb;
    int file_nd = 0, file_nrow = 0, file_ncol = 0;
    std::vector<double> file;

    void eval(double* V, const double* r, double t) const {
        switch (kind) {
        case QR_POT_HARMONIC: { // :152-161
            double sum = 0;
            for (int i = 0; i < nd; ++i) sum = sum + (r[i] * r[i]) * (0.5 * prm[i]);
            V[0] = sum;
            break;
        }
        case QR_POT_TIME_LINEAR: { // :189-201
            double a = prm[0], g = prm[1];
            double v00 = (t - a) * a;
            V[0] = v00;
            V[1] = g;
            V[2] = g;
            V[3] = -v00;
            break;
        }
        case QR_POT_TULLY_1: { // :231-247
            double A = prm[0], B = prm[1], C = prm[2], D = prm[3], x = r[0];
            double sg = x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0);
            double v00 = ((-std::exp(-(std::fabs(x) * B)) + 1.0) * A) * sg;
            double v01 = std::exp(-((x * x) * D)) * C;
            V[0] = v00;
            V[1] = v01;
            V[2] = v01;
            V[3] = -v00;
            break;
        }
        case QR_POT_TULLY_2: { // :279-297
            double A = prm[0], B = prm[1], C = prm[2], D = prm[3], E0 = prm[4], x = r[0];
            double v01 = std::exp(-((x * x) * D)) * C;
            double v11 = -(std::exp(-((x * x) * B)) * A) + E0;
            V[0] = 0.0;
            V[1] = v01;
            V[2] = v01;
            V[3] = v11;
            break;
        }
        case QR_POT_TULLY_3: { // :329-344
            double A = prm[0], B = prm[1], C = prm[2], x = r[0];
            double sg = x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0);
            double v01 = ((1.0 - std::exp(-(std::fabs(x) * C))) * sg + 1.0) * B;
            V[0] = A;
            V[1] = v01;
            V[2] = v01;
            V[3] = -A;
            break;
        }
        case QR_POT_CUSTOM: // :409-412
            for (int i = 0; i < ns * ns; ++i) V[i] = compile_eval(i, r, t);
            break;
        case QR_POT_LVC: { // :523-558
            const double h = 6.62607015e-34, e = 1.602176634e-19, c = 299792458.0, Eh = 4.3597447222060e-18;
            const double CM2EV = (1e2 * h * c) / e, EV2AU = e / Eh;
            int nm = (int)freq.size();
            double v0 = 0;
            for (int i = 0; i < nm; ++i) v0 = v0 + (r[i] * r[i]) * (0.5 * freq[i] * CM2EV);
            for (int n = 0; n < ns; ++n) {
                double term = exc[n];
                for (int i = 0; i < nm; ++i) term = term + r[i] * kap[n * nm + i];
                V[n * ns + n] = v0 + term;
            }
            for (int m = 0; m < ns; ++m)
                for (int n = m + 1; n < ns; ++n) {
                    double term = 0;
                    for (int i = 0; i < nm; ++i) term = term + r[i] * lmb[(m * ns + n) * nm + i];
                    V[m * ns + n] = term;
                    V[n * ns + m] = term;
                }
            for (int i = 0; i < ns * ns; ++i) V[i] = V[i] * EV2AU;
            break;
        }
        case QR_POT_FILE: // :470-476
            for (int col = 0; col < ns * ns; ++col) V[col] = lerp(file_nd + col, r);
            break;
        }
    }
    double compile_eval(int i, const double* r, double t) const { return ::eval(ex[i].get(), r, t); }
    // src/potential.zig:578-615
    double lerp(int column, const double* r) const {
        int nr = file_nd;
        size_t size = (size_t)std::llround(std::pow((double)file_nrow, 1.0 / (double)nr));
        auto at = [&](size_t row, int col) { return file[row * (size_t)file_ncol + col]; };
        double result = 0;
        for (size_t i = 0; i < (size_t(1) << nr); ++i) {
            double w = 1;
            size_t j = 0;
            for (int k = 0; k < nr; ++k) {
                size_t stride = 1;
                for (int q = 0; q < nr - k - 1; ++q) stride *= size;
                size_t low = 0, high = size, mid = size / 2;
                while (low < high) {
                    if (at(mid * stride, k) <= r[k]) low = mid + 1;
                    else high = mid;
                    mid = (low + high) / 2;
                }
                size_t idx = std::min(std::max(low, (size_t)1), size - 1);
                double x0 = at((idx - 1) * stride, k), x1 = at(idx * stride, k);
                double wgh = (r[k] - x0) * (1 / (x1 - x0));
                bool upper = ((i >> (nr - k - 1)) & 1) == 1;
                double wm = upper ? wgh : 1.0 - wgh;
                w = w * wm;
                j = j + (upper ? idx : idx - 1) * stride;
            }
            result = result + w * at(j, column);
        }
        return result;
    }
};

// ---------------------------------------------------------------- simulation
struct Obs {
    std::vector<double> pos, mom, pop;
    bool has_pos = false, has_mom = false, has_pop = false;
    bool has_acf = false, has_epot = false, has_ekin = false, has_norm = false;
    cplx acf{0, 0};
    double epot = NAN, ekin = NAN, norm = NAN;
};

struct Hist {
    size_t rows = 0;
    std::vector<double> pos, mom, pop, epot, ekin, etot, norm, acf;
    std::vector<double> wfn;
};

struct SolveOut {
    Obs fin;
    Hist hist;
    std::vector<cplx> psi;
    std::vector<double> acfpad, sigma; // acfpad complex interleaved
};

struct Sim {
    const qr_options& o;
    int d, S;
    size_t n, N;
    int nth;
    Potential pot;
    // Grid (wavepacket.zig:26-85)
    std::vector<double> r, k;
    double dr = 1, dk = 1;
    // Hamiltonian (wavepacket.zig:88-170)
    std::vector<double> V, W, U, K;
    // Propagator (quantum_dynamics.zig:378-536)
    std::vector<cplx> R, Kexp;
    std::vector<double> capw;
    cplx dt;
    std::vector<double> pop_apabs;
    std::vector<cplx> psi;
    std::vector<std::vector<cplx>> orthw;
    std::unique_ptr<FftNd> fft;

    explicit Sim(const qr_options& opt) : o(opt) {}

    void grid_init() { // wavepacket.zig:35-77
        d = o.ndim;
        n = o.npoint;
        N = 1;
        for (int i = 0; i < d; ++i) N *= n;
        r.assign(N * d, 0);
        k.assign(N * d, 0);
        dr = 1;
        for (int i = 0; i < d; ++i) dr *= (o.bounds[2 * i + 1] - o.bounds[2 * i]) / (double)n;
        dk = dr / (double)N;
        for (size_t i = 0; i < N; ++i) {
            size_t temp = i;
            for (int l = 0; l < d; ++l) {
                int j = d - l - 1;
                double nn = (double)(temp % n);
                double mn = o.bounds[2 * j], mx = o.bounds[2 * j + 1];
                r[i * d + j] = mn + nn * (mx - mn) / (double)n;
                double dki = 2 * M_PI / (mx - mn);
                k[i * d + j] = ((temp % n) < n / 2 ? nn : nn - (double)n) * dki;
                temp /= n;
            }
        }
    }

    void ham_update(double t) { // wavepacket.zig:137-168
        std::vector<double> Uprev;
        bool have_prev = pot.td && t > 0;
        if (have_prev) Uprev = U;
#pragma omp parallel for num_threads(nth) if (nth > 1) schedule(static)
        for (size_t i = 0; i < N; ++i) {
            pot.eval(&V[i * S * S], &r[i * d], t);
            eigh_any(S, &V[i * S * S], &W[i * S], &U[i * S * S]);
        }
        if (d == 1)
            for (size_t i = 1; i < N; ++i)
                for (int j = 0; j < S; ++j) {
                    double ov = 0;
                    for (int kk = 0; kk < S; ++kk) ov += U[i * S * S + kk * S + j] * U[(i - 1) * S * S + kk * S + j];
                    if (ov < 0)
                        for (int kk = 0; kk < S; ++kk) U[i * S * S + kk * S + j] = -U[i * S * S + kk * S + j];
                }
        if (have_prev)
            for (int j = 0; j < S; ++j) {
                double tot = 0;
                for (size_t i = 0; i < N; ++i)
                    for (int kk = 0; kk < S; ++kk) tot += U[i * S * S + kk * S + j] * Uprev[i * S * S + kk * S + j];
                if (tot < 0)
                    for (size_t i = 0; i < N; ++i)
                        for (int kk = 0; kk < S; ++kk) U[i * S * S + kk * S + j] = -U[i * S * S + kk * S + j];
            }
    }

    void ham_init() { // wavepacket.zig:96-126
        V.assign(N * S * S, 0);
        U.assign(N * S * S, 0);
        W.assign(N * S, 0);
        K.assign(N, 0);
        for (size_t i = 0; i < N; ++i) {
            double sum = 0;
            for (int j = 0; j < d; ++j) {
                double kij = k[i * d + j];
                sum += 0.5 * kij * kij / o.mass[j];
            }
            K[i] = sum;
        }
        ham_update(0);
    }

    void prop_update() { // quantum_dynamics.zig:430-468
        double dtmag = std::hypot(dt.re, dt.im);
#pragma omp parallel for num_threads(nth) if (nth > 1) schedule(static)
        for (size_t i = 0; i < N; ++i) {
            double cap_sum = 0;
            if (o.has_cap)
                for (int j = 0; j < d; ++j) {
                    double rv = r[i * d + j];
                    double dist = std::max(0.0, std::max(o.cap_bounds[2 * j] - rv, rv - o.cap_bounds[2 * j + 1]));
                    if (dist > 0) cap_sum += std::exp(o.cap_exponent * dist) - 1;
                }
            double decay = std::exp(-0.5 * cap_sum * dtmag);
            capw[i] = 1 - decay * decay;
            for (int kk = 0; kk < S; ++kk)
                for (int j = 0; j < S; ++j) {
                    cplx sum{0, 0};
                    for (int m = 0; m < S; ++m) {
                        double ukm = U[i * S * S + kk * S + m], ujm = U[i * S * S + j * S + m];
                        cplx ph = cexp_(cmul({0, -0.5 * W[i * S + m]}, dt));
                        sum = cadd(sum, {ph.re * ukm * ujm, ph.im * ukm * ujm});
                    }
                    R[i * S * S + kk * S + j] = cmul(sum, {decay, 0});
                }
        }
    }

    void prop_init() { // quantum_dynamics.zig:387-406
        R.assign(N * S * S, {0, 0});
        Kexp.assign(N, {0, 0});
        capw.assign(N, 0);
        for (size_t i = 0; i < N; ++i) Kexp[i] = cexp_(cmul({0, -K[i]}, dt));
        prop_update();
    }

    cplx* row(int s) { return &psi[(size_t)s * N]; }

    void fft_all(int sign) { // wavepacket.zig:249-255
        for (int s = 0; s < S; ++s) fft->execute(row(s), sign, nth);
    }

    void applyR() { // quantum_dynamics.zig:515-534
#pragma omp parallel for num_threads(nth) if (nth > 1) schedule(static)
        for (size_t j = 0; j < N; ++j) {
            cplx tmp[16];
            std::vector<cplx> big;
            cplx* t = tmp;
            if (S > 16) {
                big.resize(S);
                t = big.data();
            }
            for (int i = 0; i < S; ++i) {
                cplx sum{0, 0};
                for (int kk = 0; kk < S; ++kk) sum = cadd(sum, cmul(R[j * S * S + i * S + kk], psi[(size_t)kk * N + j]));
                t[i] = sum;
            }
            for (int i = 0; i < S; ++i) psi[(size_t)i * N + j] = t[i];
        }
    }

    void applyK() { // quantum_dynamics.zig:502-512
        fft_all(-1);
        for (int i = 0; i < S; ++i) {
            cplx* x = row(i);
#pragma omp parallel for num_threads(nth) if (nth > 1) schedule(static)
            for (size_t j = 0; j < N; ++j) x[j] = cmul(Kexp[j], x[j]);
        }
        fft_all(1);
    }

    void accumAbsorbed(bool adia) { // quantum_dynamics.zig:471-499
        for (int i = 0; i < S; ++i) {
            double sum = 0;
            for (size_t j = 0; j < N; ++j) {
                double w = capw[j];
                if (adia) {
                    double are = 0, aim = 0;
                    for (int kk = 0; kk < S; ++kk) {
                        double u = U[j * S * S + kk * S + i];
                        are += psi[(size_t)kk * N + j].re * u;
                        aim += psi[(size_t)kk * N + j].im * u;
                    }
                    sum += w * (are * are + aim * aim);
                } else {
                    sum += w * sqmag(psi[(size_t)i * N + j]);
                }
            }
            pop_apabs[i] += sum * dr;
        }
    }

    void step(bool adia, bool track) { // quantum_dynamics.zig:417-427
        if (track) accumAbsorbed(adia);
        applyR();
        applyK();
        if (track) accumAbsorbed(adia);
        applyR();
    }

    // wavepacket.zig observables
    double norm() const {
        double v = 0;
        for (int i = 0; i < S; ++i)
            for (size_t j = 0; j < N; ++j) v += sqmag(psi[(size_t)i * N + j]);
        return v * dr;
    }
    void normalize() { // :282-284
        double s = std::sqrt(norm());
        for (auto& z : psi) z = cdiv(z, {s, 0});
    }
    static cplx overlap(const std::vector<cplx>& a, const std::vector<cplx>& b, double dr) { // :287-295
        cplx v{0, 0};
        for (size_t i = 0; i < a.size(); ++i) v = cadd(v, cmul(cconj(a[i]), b[i]));
        return cmul(v, {dr, 0});
    }
    void setGaussian() { // :355-371
        std::fill(psi.begin(), psi.end(), cplx{0, 0});
        if (o.ic_wavefunction) { // chaining extension: the given state instead of the Gaussian
            for (size_t e = 0; e < (size_t)S * N; ++e) psi[e] = {o.ic_wavefunction[2 * e], o.ic_wavefunction[2 * e + 1]};
            normalize();
            return;
        }
        for (size_t i = 0; i < N; ++i) {
            cplx ex{0, 0};
            for (int j = 0; j < d; ++j) {
                double dx = r[i * d + j] - o.ic_position[j];
                ex = cadd(ex, {-0.5 * o.ic_gamma[j] * dx * dx, o.ic_momentum[j] * dx});
            }
            psi[(size_t)o.ic_state * N + i] = cexp_(ex);
        }
        normalize();
    }
    void toDia() { // :398-419
        std::vector<cplx> tmp(S);
        for (size_t j = 0; j < N; ++j) {
            for (int i = 0; i < S; ++i) tmp[i] = psi[(size_t)i * N + j];
            for (int i = 0; i < S; ++i) {
                cplx sum{0, 0};
                for (int kk = 0; kk < S; ++kk) sum = cadd(sum, cmul(tmp[kk], {U[j * S * S + i * S + kk], 0}));
                psi[(size_t)i * N + j] = sum;
            }
        }
    }
    void toAdia() { // :374-395
        std::vector<cplx> tmp(S);
        for (size_t j = 0; j < N; ++j) {
            for (int i = 0; i < S; ++i) tmp[i] = psi[(size_t)i * N + j];
            for (int i = 0; i < S; ++i) {
                cplx sum{0, 0};
                for (int kk = 0; kk < S; ++kk) sum = cadd(sum, cmul(tmp[kk], {U[j * S * S + kk * S + i], 0}));
                psi[(size_t)i * N + j] = sum;
            }
        }
    }

    // Observables.init, quantum_dynamics.zig:295-366
    Obs observe(const std::vector<cplx>* wfn0, unsigned wm, bool adia, bool log) {
        Obs ob;
        bool c_pos = log || (wm & QR_W_POS), c_mom = log || (wm & QR_W_MOM), c_pop = log || (wm & QR_W_POP);
        bool c_norm = log || (wm & QR_W_NORM), c_ekin = log || (wm & QR_W_EKIN), c_epot = log || (wm & QR_W_EPOT);
        if (wfn0) {
            ob.acf = overlap(*wfn0, psi, dr);
            ob.has_acf = true;
        }
        c_ekin = c_ekin || (wm & QR_W_ETOT);
        c_epot = c_epot || (wm & QR_W_ETOT);
        if (c_pos) { // :342-352
            ob.pos.assign(d, 0);
            for (int i = 0; i < S; ++i)
                for (size_t j = 0; j < N; ++j) {
                    double m2 = sqmag(psi[(size_t)i * N + j]);
                    for (int kk = 0; kk < d; ++kk) ob.pos[kk] += m2 * r[j * d + kk];
                }
            for (auto& v : ob.pos) v *= dr;
            ob.has_pos = true;
        }
        if (c_norm) {
            ob.norm = norm();
            ob.has_norm = true;
        }
        if (c_epot) { // :235-246
            double v = 0;
            for (int i = 0; i < S; ++i)
                for (int kk = 0; kk < S; ++kk)
                    for (size_t j = 0; j < N; ++j) {
                        cplx a = psi[(size_t)i * N + j], b = psi[(size_t)kk * N + j];
                        v += (a.re * b.re + a.im * b.im) * V[j * S * S + i * S + kk];
                    }
            ob.epot = v * dr;
            ob.has_epot = true;
        }
        if (c_pop) {
            ob.pop.assign(S, 0);
            if (adia) { // :317-339
                for (int i = 0; i < S; ++i)
                    for (size_t j = 0; j < N; ++j) {
                        double are = 0, aim = 0;
                        for (int kk = 0; kk < S; ++kk) {
                            double u = U[j * S * S + kk * S + i];
                            are += psi[(size_t)kk * N + j].re * u;
                            aim += psi[(size_t)kk * N + j].im * u;
                        }
                        ob.pop[i] += are * are + aim * aim;
                    }
                for (auto& v : ob.pop) v *= dr;
            } else { // :298-314
                for (int i = 0; i < S; ++i) {
                    double sum = 0;
                    for (size_t j = 0; j < N; ++j) sum += sqmag(psi[(size_t)i * N + j]);
                    ob.pop[i] = sum;
                }
                for (auto& v : ob.pop) v *= dr;
            }
            for (int j = 0; j < S; ++j) ob.pop[j] += pop_apabs[j];
            ob.has_pop = true;
        }
        if (c_mom || c_ekin) { // :347-363
            fft_all(-1);
            if (c_mom) { // :258-268
                ob.mom.assign(d, 0);
                for (int i = 0; i < S; ++i)
                    for (size_t j = 0; j < N; ++j) {
                        double m2 = sqmag(psi[(size_t)i * N + j]);
                        for (int kk = 0; kk < d; ++kk) ob.mom[kk] += m2 * k[j * d + kk];
                    }
                for (auto& v : ob.mom) v *= dk;
                ob.has_mom = true;
            }
            if (c_ekin) { // :224-232
                double v = 0;
                for (int i = 0; i < S; ++i)
                    for (size_t j = 0; j < N; ++j) v += sqmag(psi[(size_t)i * N + j]) * K[j];
                ob.ekin = v * dk;
                ob.has_ekin = true;
            }
            fft_all(1);
        }
        return ob;
    }

    // quantum_dynamics.zig:860-950
    SolveOut solve(int eig) {
        SolveOut out;
        bool itp = o.imag_nstate > 0;
        unsigned wm = o.write_mask;
        setGaussian();
        std::fill(pop_apabs.begin(), pop_apabs.end(), 0.0);
        bool calc_acf = o.has_spectrum || (wm & QR_W_ACF);
        size_t iters = (size_t)o.iterations + 1;
        Hist& h = out.hist;
        if (o.ic_adiabatic) toDia();
        bool track = o.has_cap && o.cap_track_population;
        std::vector<cplx> wfn0;
        if (calc_acf) wfn0 = psi;
        (void)eig;
        for (size_t i = 0; i < iters; ++i) {
            double time = ((double)i - 0.5) * o.time_step;
            if (i > 0 && pot.td) {
                ham_update(time);
                prop_update();
            }
            if (i > 0) step(o.adiabatic != 0, track);
            if (itp)
                for (auto& w : orthw) {
                    cplx ov = overlap(w, psi, dr);
                    for (size_t q = 0; q < psi.size(); ++q) psi[q] = csub(psi[q], cmul(ov, w[q]));
                }
            if (itp) normalize();
            if (pot.td) ham_update((double)i * o.time_step);
            Obs ob = observe(calc_acf ? &wfn0 : nullptr, wm, o.adiabatic != 0, false);
            if ((wm & QR_W_WFN) && o.adiabatic) toAdia();
            // History.append, quantum_dynamics.zig:174-215
            if (wm & QR_W_WFN) {
                for (int s = 0; s < S; ++s)
                    for (size_t j = 0; j < N; ++j) {
                        h.wfn.push_back(psi[(size_t)s * N + j].re);
                        h.wfn.push_back(psi[(size_t)s * N + j].im);
                    }
            }
            if (wm & QR_W_POS) h.pos.insert(h.pos.end(), ob.pos.begin(), ob.pos.end());
            if (wm & QR_W_MOM) h.mom.insert(h.mom.end(), ob.mom.begin(), ob.mom.end());
            if (wm & QR_W_POP) h.pop.insert(h.pop.end(), ob.pop.begin(), ob.pop.end());
            if ((wm & QR_W_EPOT) || (wm & QR_W_ETOT)) h.epot.push_back(ob.epot);
            if ((wm & QR_W_EKIN) || (wm & QR_W_ETOT)) h.ekin.push_back(ob.ekin);
            if (wm & QR_W_NORM) h.norm.push_back(ob.norm);
            if (wm & QR_W_ETOT) h.etot.push_back(ob.ekin + ob.epot);
            if (calc_acf) {
                h.acf.push_back(ob.acf.re);
                h.acf.push_back(ob.acf.im);
            }
            h.rows++;
            if ((wm & QR_W_WFN) && o.adiabatic) toDia();
            if (o.has_cap && o.cap_has_stop_norm) {
                double nm = norm();
                if (nm < o.cap_stop_norm) break;
            }
        }
        if (o.has_spectrum) spectrum(h, out);
        out.fin = observe(calc_acf ? &wfn0 : nullptr, wm, o.adiabatic != 0, true);
        out.psi = psi;
        return out;
    }

    // spectral_analysis.zig:13-44
    void spectrum(const Hist& h, SolveOut& out) {
        size_t L = h.rows;
        double decay = -std::log(o.spectrum_threshold);
        size_t lp = L + o.spectrum_padding;
        size_t ns = (lp - 1) * 2;
        out.acfpad.assign(2 * lp, 0.0);
        for (size_t i = 0; i < L; ++i) {
            double x = (double)i / (double)L;
            double window = std::exp(-decay * x * x);
            out.acfpad[2 * i] = h.acf[2 * i] * window;
            out.acfpad[2 * i + 1] = h.acf[2 * i + 1] * window;
        }
        out.sigma.assign(ns, 0.0);
        if (ns == 0) return;
        std::vector<cplx> X(ns, {0, 0});
        for (size_t kq = 0; kq < lp && kq < ns; ++kq) X[kq] = {out.acfpad[2 * kq], out.acfpad[2 * kq + 1]};
        X[0].im = 0;
        if (ns / 2 < lp) X[ns / 2].im = 0;
        for (size_t kq = 1; kq < ns / 2; ++kq) X[ns - kq] = cconj(X[kq]);
        Fft1 f(ns);
        f.run(X.data(), +1);
        for (size_t i = 0; i < ns; ++i) out.sigma[i] = X[i].re;
        double dts = o.time_step;
        for (size_t i = 0; i < ns / 2; ++i) {
            size_t j = i + ns / 2;
            double tmp = out.sigma[i];
            out.sigma[i] = out.sigma[j] * dts;
            out.sigma[j] = tmp * dts;
        }
    }
};

// quantum_dynamics.zig:606-710 plus the shape checks the reference leaves to asserts
bool check_input(const qr_options& o, int pnd, int pns) {
    auto bad = [](const char* m) {
        g_err = m;
        return false;
    };
    if (!(o.time_step > 0)) return bad("TIME STEP MUST BE GREATER THAN 0");
    for (int i = 0; i < o.ndim; ++i)
        if (!(o.mass[i] > 0)) return bad("MASS MUST BE GREATER THAN 0");
    if (o.log_interval == 0) return bad("LOG INTERVAL MUST BE GREATER THAN 0");
    if (o.npoint == 0) return bad("GRID POINT COUNT MUST BE GREATER THAN 0");
    if (o.ndim <= 0) return bad("GRID BOUNDS MUST NOT BE EMPTY");
    for (int i = 0; i < o.ndim; ++i)
        if (o.bounds[2 * i] >= o.bounds[2 * i + 1]) return bad("GRID BOUNDS MIN MUST BE LESS THAN MAX");
    if (o.has_cap) {
        for (int i = 0; i < o.ndim; ++i) {
            double c0 = o.cap_bounds[2 * i], c1 = o.cap_bounds[2 * i + 1];
            if (c0 < o.bounds[2 * i] || c1 > o.bounds[2 * i + 1] || c0 >= c1)
                return bad("ABSORBING POTENTIAL BOUNDS MUST LIE WITHIN GRID BOUNDS AND CB[0] < CB[1]");
        }
        if (!(o.cap_exponent > 0)) return bad("ABSORBING POTENTIAL EXPONENT MUST BE GREATER THAN 0");
        if (o.cap_has_stop_norm && (o.cap_stop_norm <= 0 || o.cap_stop_norm >= 1))
            return bad("ABSORBING POTENTIAL STOP_NORM MUST BE BETWEEN 0 AND 1");
    }
    if (o.has_spectrum && (o.spectrum_threshold <= 0 || o.spectrum_threshold >= 1))
        return bad("SPECTRUM THRESHOLD MUST BE BETWEEN 0 AND 1");
    if (pnd != o.ndim) return bad("POTENTIAL DIMENSION DOES NOT MATCH GRID DIMENSION");
    if ((int)o.ic_state >= pns) return bad("INITIAL STATE INDEX OUT OF RANGE");
    return true;
}

} // namespace

struct qr_result {
    int d = 0, S = 0;
    size_t N = 0;
    std::vector<SolveOut> solves;
};

extern "C" {

const char* qr_last_error(void) { return g_err.c_str(); }

int qr_run(const qr_options* opt, qr_result** out) {
    *out = nullptr;
    try {
        const qr_options& o = *opt;
        Sim sim(o);
        sim.nth = o.nthreads > 0 ? o.nthreads : 1;
        Potential& p = sim.pot;
        p.kind = o.pot.kind;
        switch (p.kind) {
        case QR_POT_HARMONIC:
            p.prm.assign(o.pot.params, o.pot.params + o.pot.nparams);
            p.nd = o.pot.nparams;
            p.ns = 1;
            break;
        case QR_POT_TIME_LINEAR:
            p.prm.assign(o.pot.params, o.pot.params + 2);
            p.nd = 1;
            p.ns = 2;
            p.td = true;
            break;
        case QR_POT_TULLY_1:
        case QR_POT_TULLY_2:
        case QR_POT_TULLY_3:
            p.prm.assign(o.pot.params, o.pot.params + o.pot.nparams);
            p.nd = 1;
            p.ns = 2;
            break;
        case QR_POT_CUSTOM:
            p.nd = o.pot.custom_ndim;
            p.ns = o.pot.custom_nstate;
            p.td = o.pot.time_dependent != 0;
            for (int i = 0; i < p.ns * p.ns; ++i) {
                try {
                    p.ex.push_back(compile_expr(o.pot.exprs[i], p.nd));
                } catch (const std::exception& e) {
                    g_err = std::string("EXPRESSION COMPILATION FAILED: ") + e.what();
                    return -1;
                }
            }
            break;
        case QR_POT_LVC:
            p.nd = o.pot.lvc_nmode;
            p.ns = o.pot.lvc_nstate;
            p.freq.assign(o.pot.lvc_freq, o.pot.lvc_freq + p.nd);
            p.exc.assign(o.pot.lvc_exc, o.pot.lvc_exc + p.ns);
            p.kap.assign(o.pot.lvc_kappa, o.pot.lvc_kappa + p.ns * p.nd);
            p.lmb.assign(o.pot.lvc_lambda, o.pot.lvc_lambda + p.ns * p.ns * p.nd);
            break;
        case QR_POT_FILE: {
            p.nd = o.pot.file_ndim;
            p.file_nd = o.pot.file_ndim;
            p.file_nrow = o.pot.file_nrow;
            p.file_ncol = o.pot.file_ncol;
            int nsq = p.file_ncol - p.file_nd;
            int ns = (int)std::lround(std::sqrt((double)(nsq > 0 ? nsq : 0)));
            p.ns = ns;
            p.file.assign(o.pot.file_data, o.pot.file_data + (size_t)p.file_nrow * p.file_ncol);
            break;
        }
        default:
            g_err = "UNKNOWN POTENTIAL";
            return -1;
        }
        if (!check_input(o, p.nd, p.ns)) return -1;
        sim.S = p.ns;
        auto res = std::make_unique<qr_result>();
        // init, quantum_dynamics.zig:713-749
        sim.dt = o.imag_nstate > 0 ? cplx{0, -o.time_step} : cplx{o.time_step, 0};
        sim.grid_init();
        sim.psi.assign((size_t)sim.S * sim.N, {0, 0});
        sim.fft = std::make_unique<FftNd>(sim.d, sim.n);
        sim.ham_init();
        sim.prop_init();
        sim.pop_apabs.assign(sim.S, 0);
        res->d = sim.d;
        res->S = sim.S;
        res->N = sim.N;
        // run, quantum_dynamics.zig:582-598
        unsigned nsolve = o.imag_nstate > 0 ? o.imag_nstate : 1;
        for (unsigned i = 0; i < nsolve; ++i) {
            res->solves.push_back(sim.solve((int)i));
            if (i < o.imag_nstate) sim.orthw.push_back(sim.psi);
        }
        *out = res.release();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

void qr_free(qr_result* r) { delete r; }
int qr_nsolve(const qr_result* r) { return (int)r->solves.size(); }
int qr_nstate(const qr_result* r) { return r->S; }
int qr_ndim(const qr_result* r) { return r->d; }
size_t qr_npoint_total(const qr_result* r) { return r->N; }

void qr_final(const qr_result* r, int s, double* pos, double* mom, double* pop, double* epot, double* ekin,
              double* norm, double* acf) {
    const Obs& o = r->solves[s].fin;
    if (pos) for (int i = 0; i < r->d; ++i) pos[i] = o.pos[i];
    if (mom) for (int i = 0; i < r->d; ++i) mom[i] = o.mom[i];
    if (pop) for (int i = 0; i < r->S; ++i) pop[i] = o.pop[i];
    if (epot) *epot = o.epot;
    if (ekin) *ekin = o.ekin;
    if (norm) *norm = o.norm;
    if (acf) {
        acf[0] = o.has_acf ? o.acf.re : NAN;
        acf[1] = o.has_acf ? o.acf.im : NAN;
    }
}

size_t qr_hist_rows(const qr_result* r, int s) { return r->solves[s].hist.rows; }

int qr_hist(const qr_result* r, int s, const char* name, double* out) {
    const Hist& h = r->solves[s].hist;
    const std::vector<double>* v = nullptr;
    int cols = 1;
    std::string n(name);
    if (n == "pos") v = &h.pos, cols = r->d;
    else if (n == "mom") v = &h.mom, cols = r->d;
    else if (n == "pop") v = &h.pop, cols = r->S;
    else if (n == "epot") v = &h.epot;
    else if (n == "ekin") v = &h.ekin;
    else if (n == "etot") v = &h.etot;
    else if (n == "norm") v = &h.norm;
    else if (n == "acf") v = &h.acf, cols = 2;
    else if (n == "wfn") v = &h.wfn, cols = (int)(2 * r->S * r->N);
    else return -1;
    if (v->empty()) return -1;
    if (out) std::copy(v->begin(), v->end(), out);
    return cols;
}

void qr_wavefunction(const qr_result* r, int s, double* out) {
    const auto& p = r->solves[s].psi;
    for (size_t i = 0; i < p.size(); ++i) {
        out[2 * i] = p[i].re;
        out[2 * i + 1] = p[i].im;
    }
}

size_t qr_spectrum_len(const qr_result* r, int s, size_t* acf_padded_len) {
    const auto& so = r->solves[s];
    if (acf_padded_len) *acf_padded_len = so.acfpad.size() / 2;
    return so.sigma.size();
}

void qr_spectrum(const qr_result* r, int s, double* acf_padded, double* sigma) {
    const auto& so = r->solves[s];
    if (acf_padded) std::copy(so.acfpad.begin(), so.acfpad.end(), acf_padded);
    if (sigma) std::copy(so.sigma.begin(), so.sigma.end(), sigma);
}

void qr_eigh(int n, const double* V, double* W, double* U) { eigh_any(n, V, W, U); }

void qr_fft(int ndim, const int* shape, int sign, double* data) {
    // square grids only (the reference uses the same npoint on every axis)
    FftNd f(ndim, (size_t)shape[0]);
    f.execute(reinterpret_cast<cplx*>(data), sign, 1);
}

int qr_expr_eval(const char* expr, int nvar, const double* vars, double t, double* value) {
    try {
        auto e = compile_expr(expr, nvar);
        *value = eval(e.get(), vars, t);
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

} // extern "C"
