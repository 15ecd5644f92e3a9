// expr.cpp -- recursive-descent compiler of potential expressions.
//
// Grammar (the ExprTk subset Zinq inputs use, src/exprtk.cpp:13-21):
//   cmp      := sum (('<'|'<='|'>'|'>='|'=='|'='|'!='|'<>') sum)*
//   sum      := product (('+'|'-') product)*
//   product  := unary (('*'|'/'|'%') unary | <implicit multiplication>)*
//   unary    := ('-'|'+') unary | power
//   power    := primary ('^' signed)*          (left-associative)
//   signed   := ('-'|'+') signed | primary
//   primary  := number | r<k> | t | pi | epsilon | inf | '(' cmp ')' | name '(' args ')'
// A constant integer exponent |p| <= 64 compiles to OP_IPOW (binary powering),
// any other exponent to pow().
#include "expr.h"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>

namespace zqd {
namespace {

struct Ast {
    uint32_t op;
    int32_t arg = 0;
    double value = 0;
    std::vector<std::unique_ptr<Ast>> kids;
};
using P = std::unique_ptr<Ast>;

P leaf(uint32_t op, int32_t arg = 0, double v = 0) {
    P a(new Ast);
    a->op = op;
    a->arg = arg;
    a->value = v;
    return a;
}
P node(uint32_t op, P x, P y = nullptr, int32_t arg = 0) {
    P a(new Ast);
    a->op = op;
    a->arg = arg;
    a->kids.push_back(std::move(x));
    if (y) a->kids.push_back(std::move(y));
    return a;
}

struct Compiler {
    const std::string& s;
    size_t p = 0;
    int nvar;
    bool implicit_ok = false; // last primary may be followed by implicit multiplication
    bool uses_time = false;

    Compiler(const std::string& text, int nv) : s(text), nvar(nv) {}

    [[noreturn]] void fail(const std::string& m) { throw std::runtime_error(m + " (at offset " + std::to_string(p) + ")"); }
    void skip() {
        while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
    }
    bool take(const char* tok) {
        skip();
        size_t n = std::strlen(tok);
        if (s.compare(p, n, tok) == 0) {
            p += n;
            return true;
        }
        return false;
    }

    P cmp() {
        P a = sum();
        for (;;) {
            uint32_t op;
            if (take("<=")) op = OP_LE;
            else if (take(">=")) op = OP_GE;
            else if (take("==")) op = OP_EQ;
            else if (take("!=") || take("<>")) op = OP_NE;
            else if (take("<")) op = OP_LT;
            else if (take(">")) op = OP_GT;
            else if (take("=")) op = OP_EQ;
            else return a;
            a = node(op, std::move(a), sum());
        }
    }
    P sum() {
        P a = product();
        for (;;) {
            if (take("+")) a = node(OP_ADD, std::move(a), product());
            else if (take("-")) a = node(OP_SUB, std::move(a), product());
            else return a;
        }
    }
    P product() {
        P a = unary();
        for (;;) {
            if (take("*")) a = node(OP_MUL, std::move(a), unary());
            else if (take("/")) a = node(OP_DIV, std::move(a), unary());
            else if (take("%")) a = node(OP_MOD, std::move(a), unary());
            else {
                skip();
                bool next_starts_operand = p < s.size() && (std::isalpha((unsigned char)s[p]) || s[p] == '(');
                if (next_starts_operand && implicit_ok) {
                    implicit_ok = false;
                    a = node(OP_MUL, std::move(a), unary());
                } else {
                    return a;
                }
            }
        }
    }
    P unary() {
        if (take("-")) return node(OP_NEG, unary());
        if (take("+")) return unary();
        return power();
    }
    P signed_operand() {
        if (take("-")) return node(OP_NEG, signed_operand());
        if (take("+")) return signed_operand();
        return primary();
    }
    static P make_power(P base, P expo) {
        const Ast* e = expo.get();
        double sgn = 1;
        while (e->op == OP_NEG) {
            sgn = -sgn;
            e = e->kids[0].get();
        }
        if (e->op == OP_CONST) {
            double v = sgn * e->value;
            if (v == std::floor(v) && std::fabs(v) <= 64) return node(OP_IPOW, std::move(base), nullptr, (int32_t)v);
        }
        return node(OP_POW, std::move(base), std::move(expo));
    }
    P power() {
        P a = primary();
        while (take("^")) a = make_power(std::move(a), signed_operand());
        return a;
    }
    P primary() {
        skip();
        implicit_ok = false;
        if (p >= s.size()) fail("unexpected end of expression");
        char c = s[p];
        if (c == '(') {
            ++p;
            P e = cmp();
            if (!take(")")) fail("missing ')'");
            implicit_ok = true;
            return e;
        }
        if (std::isdigit((unsigned char)c) || c == '.') {
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
            std::string lit = s.substr(p, q - p);
            char* end = nullptr;
            double v = std::strtod(lit.c_str(), &end);
            if (!end || *end) fail("malformed number '" + lit + "'");
            p = q;
            implicit_ok = true;
            return leaf(OP_CONST, 0, v);
        }
        if (std::isalpha((unsigned char)c) || c == '_') {
            size_t q = p;
            while (q < s.size() && (std::isalnum((unsigned char)s[q]) || s[q] == '_')) ++q;
            std::string name = s.substr(p, q - p);
            std::string lower = name;
            for (auto& ch : lower) ch = (char)std::tolower((unsigned char)ch);
            p = q;
            skip();
            if (p < s.size() && s[p] == '(') {
                ++p;
                std::vector<P> args;
                if (!take(")")) {
                    for (;;) {
                        args.push_back(cmp());
                        if (take(",")) continue;
                        if (take(")")) break;
                        fail("expected ',' or ')' in call of " + name);
                    }
                }
                implicit_ok = true;
                return call(lower, name, std::move(args));
            }
            implicit_ok = true;
            if (lower == "pi") return leaf(OP_CONST, 0, 3.141592653589793238462643383279502884);
            if (lower == "epsilon") return leaf(OP_CONST, 0, std::numeric_limits<double>::epsilon());
            if (lower == "inf") return leaf(OP_CONST, 0, std::numeric_limits<double>::infinity());
            if (name == "t") {
                uses_time = true;
                return leaf(OP_TIME);
            }
            if (name.size() >= 2 && name[0] == 'r') {
                bool digits = true;
                for (size_t i = 1; i < name.size(); ++i) digits = digits && std::isdigit((unsigned char)name[i]);
                int k = digits ? std::atoi(name.c_str() + 1) : 0;
                if (digits && k >= 1 && k <= nvar) return leaf(OP_VAR, k - 1);
            }
            fail("undefined symbol '" + name + "'");
        }
        fail(std::string("unexpected character '") + c + "'");
    }
    P call(const std::string& f, const std::string& shown, std::vector<P> args) {
        static const char* f1[F_COUNT1] = {"abs", "sgn", "exp", "log", "log10", "log2", "sqrt", "sin", "cos",
                                           "tan", "asin", "acos", "atan", "sinh", "cosh", "tanh", "erf", "erfc",
                                           "floor", "ceil", "round", "trunc", "log1p", "expm1", "cbrt"};
        static const char* f2[F_COUNT2] = {"atan2", "hypot", "fmod"};
        for (uint32_t i = 0; i < F_COUNT1; ++i)
            if (f == f1[i]) {
                if (args.size() != 1) fail(shown + " expects 1 argument");
                return node(OP_FN1, std::move(args[0]), nullptr, (int32_t)i);
            }
        if (f == "pow") {
            if (args.size() != 2) fail("pow expects 2 arguments");
            return make_power(std::move(args[0]), std::move(args[1]));
        }
        for (uint32_t i = 0; i < F_COUNT2; ++i)
            if (f == f2[i]) {
                if (args.size() != 2) fail(shown + " expects 2 arguments");
                return node(OP_FN2, std::move(args[0]), std::move(args[1]), (int32_t)i);
            }
        if (f == "min" || f == "max") {
            if (args.empty()) fail(shown + " expects arguments");
            P a(new Ast);
            a->op = f == "min" ? OP_MIN : OP_MAX;
            a->arg = (int32_t)args.size();
            a->kids = std::move(args);
            return a;
        }
        if (f == "if") {
            if (args.size() != 3) fail("if expects 3 arguments");
            P a(new Ast);
            a->op = OP_IF;
            a->kids = std::move(args);
            return a;
        }
        fail("unknown function '" + shown + "'");
    }
};

void emit(const Ast* a, ExprProgram& prog, int depth, int& maxd) {
    if (a->op == OP_CONST) {
        prog.code.push_back(enc(OP_CONST, (int32_t)prog.consts.size()));
        prog.consts.push_back(a->value);
        maxd = std::max(maxd, depth + 1);
        return;
    }
    if (a->op == OP_VAR || a->op == OP_TIME) {
        prog.code.push_back(enc(a->op, a->arg));
        maxd = std::max(maxd, depth + 1);
        return;
    }
    int d = depth;
    for (auto& k : a->kids) {
        emit(k.get(), prog, d, maxd);
        ++d;
    }
    prog.code.push_back(enc(a->op, a->arg));
}

} // namespace

bool compile_expression(const std::string& text, int nvar, ExprProgram& out, std::string& err) {
    out = ExprProgram{};
    try {
        Compiler c(text, nvar);
        P root = c.cmp();
        c.skip();
        if (c.p != text.size()) c.fail("unexpected trailing input");
        int maxd = 0;
        emit(root.get(), out, 0, maxd);
        out.code.push_back(enc(OP_END, 0));
        out.max_stack = maxd;
        out.uses_time = c.uses_time;
        if (maxd > 32) {
            err = "expression nests deeper than the 32-entry evaluation stack";
            return false;
        }
        return true;
    } catch (const std::exception& e) {
        err = e.what();
        return false;
    }
}

static double ipow_host(double x, int e) {
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

double eval_program_host(const uint32_t* code, const double* consts, const double* r, double t) {
    double st[32];
    int sp = 0;
    for (;; ++code) {
        uint32_t w = *code;
        int32_t a = arg_of(w);
        switch (op_of(w)) {
        case OP_END: return sp ? st[sp - 1] : NAN;
        case OP_CONST: st[sp++] = consts[a]; break;
        case OP_VAR: st[sp++] = r[a]; break;
        case OP_TIME: st[sp++] = t; break;
        case OP_NEG: st[sp - 1] = -st[sp - 1]; break;
        case OP_ADD: --sp; st[sp - 1] = st[sp - 1] + st[sp]; break;
        case OP_SUB: --sp; st[sp - 1] = st[sp - 1] - st[sp]; break;
        case OP_MUL: --sp; st[sp - 1] = st[sp - 1] * st[sp]; break;
        case OP_DIV: --sp; st[sp - 1] = st[sp - 1] / st[sp]; break;
        case OP_MOD: --sp; st[sp - 1] = std::fmod(st[sp - 1], st[sp]); break;
        case OP_POW: --sp; st[sp - 1] = std::pow(st[sp - 1], st[sp]); break;
        case OP_IPOW: st[sp - 1] = ipow_host(st[sp - 1], a); break;
        case OP_LT: --sp; st[sp - 1] = st[sp - 1] < st[sp] ? 1.0 : 0.0; break;
        case OP_LE: --sp; st[sp - 1] = st[sp - 1] <= st[sp] ? 1.0 : 0.0; break;
        case OP_GT: --sp; st[sp - 1] = st[sp - 1] > st[sp] ? 1.0 : 0.0; break;
        case OP_GE: --sp; st[sp - 1] = st[sp - 1] >= st[sp] ? 1.0 : 0.0; break;
        case OP_EQ: --sp; st[sp - 1] = st[sp - 1] == st[sp] ? 1.0 : 0.0; break;
        case OP_NE: --sp; st[sp - 1] = st[sp - 1] != st[sp] ? 1.0 : 0.0; break;
        case OP_IF: sp -= 2; st[sp - 1] = st[sp - 1] != 0.0 ? st[sp] : st[sp + 1]; break;
        case OP_MIN:
        case OP_MAX: {
            int n = a;
            double v = st[sp - n];
            for (int i = 1; i < n; ++i) {
                double x = st[sp - n + i];
                v = op_of(w) == OP_MIN ? (x < v ? x : v) : (x > v ? x : v);
            }
            sp -= n - 1;
            st[sp - 1] = v;
            break;
        }
        case OP_FN2: {
            --sp;
            double x = st[sp - 1], y = st[sp];
            st[sp - 1] = a == F_ATAN2 ? std::atan2(x, y) : a == F_HYPOT ? std::hypot(x, y) : std::fmod(x, y);
            break;
        }
        case OP_FN1: {
            double x = st[sp - 1], v;
            switch (a) {
            case F_ABS: v = std::fabs(x); break;
            case F_SGN: v = x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); break;
            case F_EXP: v = std::exp(x); break;
            case F_LOG: v = std::log(x); break;
            case F_LOG10: v = std::log10(x); break;
            case F_LOG2: v = std::log2(x); break;
            case F_SQRT: v = std::sqrt(x); break;
            case F_SIN: v = std::sin(x); break;
            case F_COS: v = std::cos(x); break;
            case F_TAN: v = std::tan(x); break;
            case F_ASIN: v = std::asin(x); break;
            case F_ACOS: v = std::acos(x); break;
            case F_ATAN: v = std::atan(x); break;
            case F_SINH: v = std::sinh(x); break;
            case F_COSH: v = std::cosh(x); break;
            case F_TANH: v = std::tanh(x); break;
            case F_ERF: v = std::erf(x); break;
            case F_ERFC: v = std::erfc(x); break;
            case F_FLOOR: v = std::floor(x); break;
            case F_CEIL: v = std::ceil(x); break;
            case F_ROUND: v = std::round(x); break;
            case F_TRUNC: v = std::trunc(x); break;
            case F_LOG1P: v = std::log1p(x); break;
            case F_EXPM1: v = std::expm1(x); break;
            default: v = std::cbrt(x); break;
            }
            st[sp - 1] = v;
            break;
        }
        default: return NAN;
        }
    }
}

} // namespace zqd
