/*
 * Device arithmetic of one bytecode operator, f32 and f64.
 *
 * The guards and special cases follow the reference's device interpreter
 * (my-version/src/cuda/eval.cu:404-573 `rc_exec_row`) for the f32 scoring
 * path, its fit-kernel value sweeps (eval.cu:1173-1233 `ft_forward`,
 * :1324-1381 `ft_forward_d`) and their adjoints (eval.cu:1236-1317,
 * :1383-1463), which in turn mirror the CPU `expr::eval` (my-version/src/
 * expr.rs:1054-1326) and `fit::backward_impl` (my-version/src/fit.rs:1453-1671).
 */
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

enum {
    OP_CONST = 0, OP_VAR = 1, OP_ADD = 2, OP_SUB = 3, OP_MUL = 4, OP_DIV = 5,
    OP_SIN = 6, OP_COS = 7, OP_TAN = 8, OP_EXP = 9, OP_LOG = 10, OP_SQRT = 11,
    OP_ABS = 12, OP_TANH = 13, OP_SIG = 14, OP_SQUARE = 15, OP_CUBE = 16, OP_NEG = 17,
    OP_GAUSS = 18, OP_STEP = 19, OP_POW = 20, OP_SINH = 21, OP_COSH = 22,
    OP_FLOOR = 23, OP_CEIL = 24, OP_ROUND = 25, OP_MOD = 26, OP_ATAN2 = 27,
    OP_ERF = 28, OP_ERFC = 29, OP_MIN = 30, OP_MAX = 31, OP_IF = 32, OP_SIGN = 33,
    OP_EQUAL = 34, OP_LESS = 35, OP_LESS_OR_EQUAL = 36, OP_GREATER = 37,
    OP_GREATER_OR_EQUAL = 38, OP_AND = 39, OP_OR = 40, OP_XOR = 41, OP_NOT = 42,
    OP_HALT = 255
};

/* The device stack bound of the postfix format (eval.cu:85). */
#define RC_MAX_STACK 64

__device__ __forceinline__ float rc_nanf() { return CUDART_NAN_F; }

/* One unary operator in f32 (eval.cu:530-569). Unknown codes give NaN. */
__device__ __forceinline__ float rc_unary_f(unsigned op, float a)
{
    switch (op) {
        case OP_SIN: return sinf(a);
        case OP_COS: return cosf(a);
        case OP_TAN: {
            float t = tanf(a);
            return isfinite(t) ? t : rc_nanf();
        }
        case OP_EXP: return expf(a);
        case OP_LOG: return a > 0.0f ? logf(a) : rc_nanf();
        case OP_SQRT: return a >= 0.0f ? sqrtf(a) : rc_nanf();
        case OP_ABS: return fabsf(a);
        case OP_TANH: return tanhf(a);
        case OP_SIG: return 1.0f / (1.0f + expf(-a));
        case OP_SQUARE: return a * a;
        case OP_CUBE: return a * a * a;
        case OP_NEG: return -a;
        case OP_GAUSS: return expf(-a * a);
        case OP_STEP: return a > 0.0f ? 1.0f : 0.0f;
        case OP_SINH: return sinhf(a);
        case OP_COSH: return coshf(a);
        case OP_FLOOR: return floorf(a);
        case OP_CEIL: return ceilf(a);
        case OP_ROUND: return roundf(a);
        case OP_ERF: return a == 0.0f ? 0.0f : erff(a);
        case OP_ERFC: return erfcf(a);
        case OP_SIGN:
            return isnan(a) ? rc_nanf() : (a > 0.0f ? 1.0f : (a < 0.0f ? -1.0f : 0.0f));
        case OP_NOT: return isnan(a) ? rc_nanf() : (a > 0.0f ? 0.0f : 1.0f);
        default: return rc_nanf();
    }
}

/* One binary operator in f32 (eval.cu:430-521). */
__device__ __forceinline__ float rc_binary_f(unsigned op, float a, float b)
{
    switch (op) {
        case OP_ADD: return a + b;
        case OP_SUB: return a - b;
        case OP_MUL: return a * b;
        case OP_DIV: return fabsf(b) < 1e-12f ? rc_nanf() : a / b;
        case OP_POW:
            return (a < 0.0f && fabsf(b - roundf(b)) > 1e-9f) ? rc_nanf() : powf(a, b);
        case OP_MOD: {
            float r = rc_nanf();
            if (isfinite(a) && isfinite(b) && fabsf(b) >= 1e-12f) {
                float q = a / b;
                if (isfinite(q)) {
                    r = fmaf(-b, floorf(q), a);
                    float ab = fabsf(b);
                    float rs = b > 0.0f ? r : -r;
                    if (rs < 0.0f) r += b;
                    else if (rs >= ab) r -= b;
                }
            }
            return r;
        }
        case OP_ATAN2: return (isnan(a) || isnan(b)) ? rc_nanf() : atan2f(a, b);
        case OP_MIN: return (isnan(a) || isnan(b)) ? rc_nanf() : fminf(a, b);
        case OP_MAX: return (isnan(a) || isnan(b)) ? rc_nanf() : fmaxf(a, b);
        case OP_EQUAL: return (isnan(a) || isnan(b)) ? rc_nanf() : (a == b ? 1.0f : 0.0f);
        case OP_LESS: return (isnan(a) || isnan(b)) ? rc_nanf() : (a < b ? 1.0f : 0.0f);
        case OP_LESS_OR_EQUAL:
            return (isnan(a) || isnan(b)) ? rc_nanf() : (a <= b ? 1.0f : 0.0f);
        case OP_GREATER: return (isnan(a) || isnan(b)) ? rc_nanf() : (a > b ? 1.0f : 0.0f);
        case OP_GREATER_OR_EQUAL:
            return (isnan(a) || isnan(b)) ? rc_nanf() : (a >= b ? 1.0f : 0.0f);
        case OP_AND:
            return (isnan(a) || isnan(b)) ? rc_nanf() : ((a > 0.0f && b > 0.0f) ? 1.0f : 0.0f);
        case OP_OR:
            return (isnan(a) || isnan(b)) ? rc_nanf() : ((a > 0.0f || b > 0.0f) ? 1.0f : 0.0f);
        case OP_XOR:
            return (isnan(a) || isnan(b)) ? rc_nanf() : (((a > 0.0f) != (b > 0.0f)) ? 1.0f : 0.0f);
        default: return rc_nanf();
    }
}

/* ---- fit-record value sweep: the analytic operator subset ------------- */

/* f32 value of one fit-record node from its children (eval.cu:1173-1233).
   `exp` carries the f64 path's 700 cut-off, as the reference's fit sweep does. */
__device__ __forceinline__ float ft_value_f(unsigned op, float a, float b)
{
    switch (op) {
        case OP_ADD: return a + b;
        case OP_SUB: return a - b;
        case OP_MUL: return a * b;
        case OP_DIV: return fabsf(b) < 1e-12f ? rc_nanf() : a / b;
        case OP_POW:
            return (a < 0.0f && fabsf(b - roundf(b)) > 1e-9f) ? rc_nanf() : powf(a, b);
        case OP_SIN: return sinf(a);
        case OP_COS: return cosf(a);
        case OP_TAN: {
            float t = tanf(a);
            return isfinite(t) ? t : rc_nanf();
        }
        case OP_EXP: return a > 700.0f ? CUDART_INF_F : expf(a);
        case OP_LOG: return a > 0.0f ? logf(a) : rc_nanf();
        case OP_SQRT: return a >= 0.0f ? sqrtf(a) : rc_nanf();
        case OP_ABS: return fabsf(a);
        case OP_TANH: return tanhf(a);
        case OP_SIG: return 1.0f / (1.0f + expf(-a));
        case OP_SQUARE: return a * a;
        case OP_CUBE: return a * a * a;
        case OP_NEG: return -a;
        case OP_GAUSS: return expf(-a * a);
        case OP_SINH: return sinhf(a);
        case OP_COSH: return coshf(a);
        case OP_ERF: return a == 0.0f ? 0.0f : erff(a);
        case OP_ERFC: return erfcf(a);
        default: return rc_nanf();
    }
}

/* f64 twin (eval.cu:1324-1381). */
__device__ __forceinline__ double ft_value_d(unsigned op, double a, double b)
{
    switch (op) {
        case OP_ADD: return a + b;
        case OP_SUB: return a - b;
        case OP_MUL: return a * b;
        case OP_DIV: return fabs(b) < 1e-12 ? CUDART_NAN : a / b;
        case OP_POW:
            return (a < 0.0 && fabs(b - round(b)) > 1e-9) ? CUDART_NAN : pow(a, b);
        case OP_SIN: return sin(a);
        case OP_COS: return cos(a);
        case OP_TAN: {
            double t = tan(a);
            return isfinite(t) ? t : CUDART_NAN;
        }
        case OP_EXP: return a > 700.0 ? CUDART_INF : exp(a);
        case OP_LOG: return a > 0.0 ? log(a) : CUDART_NAN;
        case OP_SQRT: return a >= 0.0 ? sqrt(a) : CUDART_NAN;
        case OP_ABS: return fabs(a);
        case OP_TANH: return tanh(a);
        case OP_SIG: return 1.0 / (1.0 + exp(-a));
        case OP_SQUARE: return a * a;
        case OP_CUBE: return a * a * a;
        case OP_NEG: return -a;
        case OP_GAUSS: return exp(-a * a);
        case OP_SINH: return sinh(a);
        case OP_COSH: return cosh(a);
        case OP_ERF: return a == 0.0 ? 0.0 : erf(a);
        case OP_ERFC: return erfc(a);
        default: return CUDART_NAN;
    }
}

/* Local partial derivatives of one node w.r.t. its operands, f32
   (eval.cu:1253-1313): d0 = d node / d a, d1 = d node / d b. A `pow` with a
   non-positive base passes nothing, as in the reference. */
__device__ __forceinline__ void ft_partials_f(unsigned op, float x, float y, float &d0, float &d1)
{
    d0 = 0.0f;
    d1 = 0.0f;
    switch (op) {
        case OP_NEG: d0 = -1.0f; break;
        case OP_EXP: d0 = expf(x); break;
        case OP_LOG: d0 = 1.0f / x; break;
        case OP_ABS: d0 = x >= 0.0f ? 1.0f : -1.0f; break;
        case OP_SQRT: d0 = 1.0f / (2.0f * sqrtf(x)); break;
        case OP_SIN: d0 = cosf(x); break;
        case OP_COS: d0 = -sinf(x); break;
        case OP_TAN: {
            float t = cosf(x);
            d0 = 1.0f / (t * t);
        } break;
        case OP_SINH: d0 = coshf(x); break;
        case OP_COSH: d0 = sinhf(x); break;
        case OP_TANH: {
            float t = tanhf(x);
            d0 = 1.0f - t * t;
        } break;
        case OP_SIG: {
            float s = 1.0f / (1.0f + expf(-x));
            d0 = s * (1.0f - s);
        } break;
        case OP_GAUSS: d0 = (-2.0f * x) * expf(-x * x); break;
        case OP_SQUARE: d0 = 2.0f * x; break;
        case OP_CUBE: d0 = 3.0f * x * x; break;
        case OP_ERF: d0 = 1.1283791670955126f * expf(-x * x); break;
        case OP_ERFC: d0 = -1.1283791670955126f * expf(-x * x); break;
        case OP_ADD: d0 = 1.0f; d1 = 1.0f; break;
        case OP_SUB: d0 = 1.0f; d1 = -1.0f; break;
        case OP_MUL: d0 = y; d1 = x; break;
        case OP_DIV: d0 = 1.0f / y; d1 = -x / (y * y); break;
        case OP_POW:
            if (x > 0.0f) {
                d0 = y * powf(x, y - 1.0f);
                d1 = powf(x, y) * logf(x);
            }
            break;
        default: break;
    }
}

/* f64 twin (eval.cu:1400-1459). */
__device__ __forceinline__ void ft_partials_d(unsigned op, double x, double y, double &d0,
                                              double &d1)
{
    d0 = 0.0;
    d1 = 0.0;
    switch (op) {
        case OP_NEG: d0 = -1.0; break;
        case OP_EXP: d0 = exp(x); break;
        case OP_LOG: d0 = 1.0 / x; break;
        case OP_ABS: d0 = x >= 0.0 ? 1.0 : -1.0; break;
        case OP_SQRT: d0 = 1.0 / (2.0 * sqrt(x)); break;
        case OP_SIN: d0 = cos(x); break;
        case OP_COS: d0 = -sin(x); break;
        case OP_TAN: {
            double t = cos(x);
            d0 = 1.0 / (t * t);
        } break;
        case OP_SINH: d0 = cosh(x); break;
        case OP_COSH: d0 = sinh(x); break;
        case OP_TANH: {
            double t = tanh(x);
            d0 = 1.0 - t * t;
        } break;
        case OP_SIG: {
            double s = 1.0 / (1.0 + exp(-x));
            d0 = s * (1.0 - s);
        } break;
        case OP_GAUSS: d0 = (-2.0 * x) * exp(-x * x); break;
        case OP_SQUARE: d0 = 2.0 * x; break;
        case OP_CUBE: d0 = 3.0 * x * x; break;
        case OP_ERF: d0 = 1.1283791670955126 * exp(-x * x); break;
        case OP_ERFC: d0 = -1.1283791670955126 * exp(-x * x); break;
        case OP_ADD: d0 = 1.0; d1 = 1.0; break;
        case OP_SUB: d0 = 1.0; d1 = -1.0; break;
        case OP_MUL: d0 = y; d1 = x; break;
        case OP_DIV: d0 = 1.0 / y; d1 = -x / (y * y); break;
        case OP_POW:
            if (x > 0.0) {
                d0 = y * pow(x, y - 1.0);
                d1 = pow(x, y) * log(x);
            }
            break;
        default: break;
    }
}

/* True for the operators a fit record may hold (fit.rs:890-920). */
__host__ __device__ __forceinline__ bool ft_op_supported(unsigned op)
{
    switch (op) {
        case OP_CONST: case OP_VAR: case OP_ADD: case OP_SUB: case OP_MUL: case OP_DIV:
        case OP_SIN: case OP_COS: case OP_TAN: case OP_EXP: case OP_LOG: case OP_SQRT:
        case OP_ABS: case OP_TANH: case OP_SIG: case OP_SQUARE: case OP_CUBE: case OP_NEG:
        case OP_GAUSS: case OP_POW: case OP_SINH: case OP_COSH: case OP_ERF: case OP_ERFC:
            return true;
        default: return false;
    }
}

__host__ __device__ __forceinline__ bool ft_op_binary(unsigned op)
{
    return op == OP_ADD || op == OP_SUB || op == OP_MUL || op == OP_DIV || op == OP_POW;
}
