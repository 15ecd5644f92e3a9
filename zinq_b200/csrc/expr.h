// expr.h -- host compiler of potential expressions into device bytecode.
//
// Replaces ExprTk in Zinq's `custom` potential (src/exprtk.cpp:10-40,
// src/potential.zig:364-451): an expression over r1..rN, t and the constants
// pi, epsilon, inf is compiled once on the host into a postfix program that
// the FP64 stack interpreter in potential.cuh evaluates per grid point.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#ifdef __CUDACC__
#define ZQD_HD __host__ __device__
#else
#define ZQD_HD
#endif

namespace zqd {

enum ExprOp : uint32_t {
    OP_END = 0,
    OP_CONST = 1, // operand: index into the constant pool
    OP_VAR = 2,   // operand: coordinate index (r1 -> 0)
    OP_TIME = 3,
    OP_NEG = 4,
    OP_ADD = 5,
    OP_SUB = 6,
    OP_MUL = 7,
    OP_DIV = 8,
    OP_MOD = 9,
    OP_POW = 10,
    OP_IPOW = 11, // operand: signed integer exponent (two's complement in 24 bits)
    OP_LT = 12,
    OP_LE = 13,
    OP_GT = 14,
    OP_GE = 15,
    OP_EQ = 16,
    OP_NE = 17,
    OP_FN1 = 18, // operand: Fn1 code
    OP_FN2 = 19, // operand: Fn2 code
    OP_MIN = 20, // operand: argument count
    OP_MAX = 21,
    OP_IF = 22,
};

enum Fn1 : uint32_t {
    F_ABS, F_SGN, F_EXP, F_LOG, F_LOG10, F_LOG2, F_SQRT, F_SIN, F_COS, F_TAN, F_ASIN, F_ACOS, F_ATAN,
    F_SINH, F_COSH, F_TANH, F_ERF, F_ERFC, F_FLOOR, F_CEIL, F_ROUND, F_TRUNC, F_LOG1P, F_EXPM1, F_CBRT,
    F_COUNT1
};
enum Fn2 : uint32_t { F_ATAN2, F_HYPOT, F_FMOD, F_COUNT2 };

inline uint32_t enc(uint32_t op, int32_t operand) { return op | ((uint32_t)(operand & 0xFFFFFF) << 8); }
ZQD_HD inline uint32_t op_of(uint32_t w) { return w & 0xFFu; }
ZQD_HD inline int32_t arg_of(uint32_t w) { return ((int32_t)w) >> 8; }

struct ExprProgram {
    std::vector<uint32_t> code; // terminated by OP_END
    std::vector<double> consts;
    int max_stack = 0;
    bool uses_time = false;
};

// Compiles text; on failure returns false and sets err.
bool compile_expression(const std::string& text, int nvar, ExprProgram& out, std::string& err);

// Host evaluation of a compiled program (used for potential_plot-like checks and tests).
double eval_program_host(const uint32_t* code, const double* consts, const double* r, double t);

} // namespace zqd
