/*
 * Device side of the batched scorer: the f32 interpreter with a running
 * first-order rounding-error bound, the per-warp deterministic accumulation,
 * the finalize pass that flags candidates whose f32 result cannot be trusted
 * to the parity tolerance, and the f64 re-check lane for those candidates.
 *
 * Operator semantics: my-version/src/cuda/eval.cu:404-573 (f32, the device
 * reference) and my-version/src/expr.rs:1054-1326 (f64, the CPU oracle the
 * re-check lane reproduces). Objectives: eval.cu:846-1088.
 */
#pragma once

#include <cuda_bf16.h>

#include "rc_internal.h"
#include "rc_ops.cuh"

/* Internal scoring modes. 0..14 are the RC_SCORE_* codes (eval.cu:609-640). */
enum {
    SM_SQUARED = 0, SM_ABSOLUTE = 1, SM_LOG_SQUASHED = 2, SM_SIGNED = 3, SM_MAXIMUM = 4,
    SM_CORRELATION = 5, SM_CORRELATION_SIGNED = 6, SM_AIC = 7, SM_AICC = 8, SM_BIC = 9,
    SM_LOG_LOSS = 10, SM_BRIER = 11, SM_HINGE_SIGMOID = 12, SM_HINGE_ORDINARY = 13,
    SM_HINGE_SQUARED = 14,
    SM_EVAL_SQUARED = 20, SM_EVAL_LOG_SQUASHED = 21, SM_EVAL_ABSOLUTE = 24,
    SM_PREDICT = 30,
    SM_CORR_PASS1 = 31, SM_CORR_PASS2 = 32
};

#define RC_SCORE_NONFINITE 2
#define RC_SCORE_ALL_ZERO_WEIGHT 4

/* Unit roundoff of a correctly rounded f32 operation, and the bound used for
   CUDA's f32 library functions (at most 4 ulp for every function used here). */
#define RC_EPS32 5.9604645e-08f
#define RC_FUN_ERR (8.0f * RC_EPS32)
/* A candidate whose accumulated loss error bound exceeds this fraction of its
   loss is rescored in f64 (ten times below the 1e-4 parity bar). */
#define RC_FLAG_TOL 1e-5

/* Rows per work-item tile, fixed so that a candidate's reduction order
   depends only on n and the kernel shape. */
#define RC_TILE_ROWS 32768

__device__ __forceinline__ bool rc_mode_tracks(int mode)
{
    return mode < SM_EVAL_SQUARED || mode == SM_CORR_PASS1 || mode == SM_CORR_PASS2;
}

/* ---- first-order error bounds ----------------------------------------- */

/* Absolute error bound of op(a) given the bound ea of its operand and the
   computed result r (which includes its own rounding). Piecewise-constant
   operators report the jump when the operand's uncertainty reaches a
   discontinuity. */
template <unsigned OPC>
__device__ __forceinline__ float rc_un_err(float a, float ea, float r)
{
    const float ar = fabsf(r);
    switch (OPC) {
        case OP_SIN: case OP_COS: case OP_TANH: return ea + RC_FUN_ERR * ar;
        case OP_TAN: return ea * (1.0f + r * r) + RC_FUN_ERR * ar;
        case OP_EXP: return ar * ea + RC_FUN_ERR * ar;
        case OP_LOG:
            if (ea == 0.0f) return RC_FUN_ERR * ar;
            return a > ea ? __fdividef(ea, a - ea) + RC_FUN_ERR * ar : CUDART_INF_F;
        case OP_SQRT:
            if (ea == 0.0f) return RC_EPS32 * ar;
            return ar > 0.0f ? __fdividef(ea, ar) + RC_EPS32 * ar : sqrtf(ea);
        case OP_ABS: case OP_NEG: return ea;
        case OP_SIG: return 0.25f * ea + RC_FUN_ERR * ar;
        case OP_SQUARE: return (2.0f * fabsf(a) + ea) * ea + RC_EPS32 * ar;
        case OP_CUBE: {
            const float aa = fabsf(a) + ea;
            return 3.0f * aa * aa * ea + 2.0f * RC_EPS32 * ar;
        }
        case OP_GAUSS: return 0.86f * ea + RC_FUN_ERR * ar; /* |d/da e^-a^2| <= sqrt(2/e) */
        case OP_SINH: case OP_COSH: return (ar + 1.0f) * ea * 1.001f + RC_FUN_ERR * ar;
        case OP_ERF: case OP_ERFC: return 1.1284f * ea + RC_FUN_ERR * ar;
        case OP_STEP: case OP_SIGN: case OP_NOT:
            return (ea > 0.0f && fabsf(a) <= ea) ? 1.0f : 0.0f;
        case OP_FLOOR: case OP_CEIL: {
            const float d = fminf(a - floorf(a), ceilf(a) - a);
            return (ea > 0.0f && d <= ea) ? 1.0f : 0.0f;
        }
        case OP_ROUND: {
            const float d = fabsf(a - floorf(a) - 0.5f);
            return (ea > 0.0f && d <= ea) ? 1.0f : 0.0f;
        }
        default: return 0.0f;
    }
}

template <unsigned OPC>
__device__ __forceinline__ float rc_bin_err(float a, float ea, float b, float eb, float r)
{
    const float ar = fabsf(r);
    switch (OPC) {
        case OP_ADD: case OP_SUB: return ea + eb + RC_EPS32 * ar;
        case OP_MUL: return fabsf(b) * ea + fabsf(a) * eb + ea * eb + RC_EPS32 * ar;
        case OP_DIV: {
            const float ab = fabsf(b);
            if (eb == 0.0f) return __fdividef(ea, ab) + RC_EPS32 * ar;
            return ab > eb ? __fdividef(ea + ar * eb, ab - eb) + RC_EPS32 * ar : CUDART_INF_F;
        }
        case OP_POW: {
            if (ea == 0.0f && eb == 0.0f) return RC_FUN_ERR * ar;
            if (a > ea) {
                const float rel = fabsf(b) * __fdividef(ea, a - ea) + fabsf(__logf(a)) * eb;
                return ar * rel * 1.001f + RC_FUN_ERR * ar;
            }
            if (a < -ea && eb == 0.0f) {
                return ar * fabsf(b) * __fdividef(ea, -a - ea) * 1.001f + RC_FUN_ERR * ar;
            }
            return CUDART_INF_F;
        }
        case OP_MOD: {
            const float ab = fabsf(b);
            const float q = __fdividef(a, b);
            const float dq = __fdividef(ea + fabsf(q) * eb, ab) + 4.0f * RC_EPS32 * fabsf(q);
            const float dist = fabsf(q - rintf(q));
            if (dist <= dq) return ab + eb;
            return ea + floorf(fabsf(q) + 1.0f) * eb + 4.0f * RC_EPS32 * (fabsf(a) + ab);
        }
        case OP_ATAN2: {
            const float d = a * a + b * b;
            if (ea == 0.0f && eb == 0.0f) return RC_FUN_ERR * ar;
            if (b < 0.0f && fabsf(a) <= ea) return 6.2832f;
            return d > 0.0f ? __fdividef(fabsf(b) * ea + fabsf(a) * eb, d) + RC_FUN_ERR * ar
                            : CUDART_INF_F;
        }
        case OP_MIN: case OP_MAX: return fmaxf(ea, eb);
        case OP_EQUAL: case OP_LESS: case OP_LESS_OR_EQUAL: case OP_GREATER:
        case OP_GREATER_OR_EQUAL:
            return (ea + eb > 0.0f && fabsf(a - b) <= ea + eb) ? 1.0f : 0.0f;
        case OP_AND: case OP_OR: case OP_XOR:
            return ((ea > 0.0f && fabsf(a) <= ea) || (eb > 0.0f && fabsf(b) <= eb)) ? 1.0f : 0.0f;
        default: return 0.0f;
    }
}

/* ---- the f32 interpreter ------------------------------------------------- */

#define RC_U4(OPC)                                                                  \
    {                                                                               \
        const float r0 = rc_unary_f(OPC, t0), r1 = rc_unary_f(OPC, t1);             \
        const float r2 = rc_unary_f(OPC, t2), r3 = rc_unary_f(OPC, t3);             \
        if (TRACK) {                                                                \
            e0 = rc_un_err<OPC>(t0, e0, r0);                                        \
            e1 = rc_un_err<OPC>(t1, e1, r1);                                        \
            e2 = rc_un_err<OPC>(t2, e2, r2);                                        \
            e3 = rc_un_err<OPC>(t3, e3, r3);                                        \
        }                                                                           \
        t0 = r0; t1 = r1; t2 = r2; t3 = r3;                                         \
    }
#define RC_B4(OPC)                                                                  \
    {                                                                               \
        const float r0 = rc_binary_f(OPC, a0, b0), r1 = rc_binary_f(OPC, a1, b1);   \
        const float r2 = rc_binary_f(OPC, a2, b2), r3 = rc_binary_f(OPC, a3, b3);   \
        if (TRACK) {                                                                \
            e0 = rc_bin_err<OPC>(a0, ea0, b0, eb0, r0);                             \
            e1 = rc_bin_err<OPC>(a1, ea1, b1, eb1, r1);                             \
            e2 = rc_bin_err<OPC>(a2, ea2, b2, eb2, r2);                             \
            e3 = rc_bin_err<OPC>(a3, ea3, b3, eb3, r3);                             \
        }                                                                           \
        t0 = r0; t1 = r1; t2 = r2; t3 = r3;                                         \
    }

/* The operators outside the common set (+, -, *, /, pow, sin, cos, exp,
   log, sqrt, square, neg) run out of line: one copy each, called with the
   thread's four values and bounds. Inlining all of them into the
   interpreter's dispatch made its code larger than the instruction cache
   holds (most stalls were "no instruction"); with them called, the scoring
   kernel takes 11 % less time on the benchmark batch, with identical bits. */
struct RcF8 {
    float t[4];
    float e[4];
};

template <bool TRACK>
__device__ __noinline__ RcF8 rc_un4_rare(unsigned op, RcF8 v)
{
    float t0 = v.t[0], t1 = v.t[1], t2 = v.t[2], t3 = v.t[3];
    float e0 = v.e[0], e1 = v.e[1], e2 = v.e[2], e3 = v.e[3];
    switch (op) {
        case OP_TAN: RC_U4(OP_TAN); break;
        case OP_ABS: RC_U4(OP_ABS); break;
        case OP_TANH: RC_U4(OP_TANH); break;
        case OP_SIG: RC_U4(OP_SIG); break;
        case OP_CUBE: RC_U4(OP_CUBE); break;
        case OP_GAUSS: RC_U4(OP_GAUSS); break;
        case OP_STEP: RC_U4(OP_STEP); break;
        case OP_SINH: RC_U4(OP_SINH); break;
        case OP_COSH: RC_U4(OP_COSH); break;
        case OP_FLOOR: RC_U4(OP_FLOOR); break;
        case OP_CEIL: RC_U4(OP_CEIL); break;
        case OP_ROUND: RC_U4(OP_ROUND); break;
        case OP_ERF: RC_U4(OP_ERF); break;
        case OP_ERFC: RC_U4(OP_ERFC); break;
        case OP_SIGN: RC_U4(OP_SIGN); break;
        case OP_NOT: RC_U4(OP_NOT); break;
        default: t0 = t1 = t2 = t3 = rc_nanf(); break;
    }
    RcF8 o;
    o.t[0] = t0; o.t[1] = t1; o.t[2] = t2; o.t[3] = t3;
    o.e[0] = e0; o.e[1] = e1; o.e[2] = e2; o.e[3] = e3;
    return o;
}

struct RcB16 {
    float a[4], b[4], ea[4], eb[4];
};

template <bool TRACK>
__device__ __noinline__ RcF8 rc_bin4_rare(unsigned op, RcB16 v)
{
    const float a0 = v.a[0], a1 = v.a[1], a2 = v.a[2], a3 = v.a[3];
    const float b0 = v.b[0], b1 = v.b[1], b2 = v.b[2], b3 = v.b[3];
    const float ea0 = v.ea[0], ea1 = v.ea[1], ea2 = v.ea[2], ea3 = v.ea[3];
    const float eb0 = v.eb[0], eb1 = v.eb[1], eb2 = v.eb[2], eb3 = v.eb[3];
    float t0, t1, t2, t3, e0 = 0.f, e1 = 0.f, e2 = 0.f, e3 = 0.f;
    switch (op) {
        case OP_MOD: RC_B4(OP_MOD); break;
        case OP_ATAN2: RC_B4(OP_ATAN2); break;
        case OP_MIN: RC_B4(OP_MIN); break;
        case OP_MAX: RC_B4(OP_MAX); break;
        case OP_EQUAL: RC_B4(OP_EQUAL); break;
        case OP_LESS: RC_B4(OP_LESS); break;
        case OP_LESS_OR_EQUAL: RC_B4(OP_LESS_OR_EQUAL); break;
        case OP_GREATER: RC_B4(OP_GREATER); break;
        case OP_GREATER_OR_EQUAL: RC_B4(OP_GREATER_OR_EQUAL); break;
        case OP_AND: RC_B4(OP_AND); break;
        case OP_OR: RC_B4(OP_OR); break;
        case OP_XOR: RC_B4(OP_XOR); break;
        default: t0 = t1 = t2 = t3 = rc_nanf(); break;
    }
    RcF8 o;
    o.t[0] = t0; o.t[1] = t1; o.t[2] = t2; o.t[3] = t3;
    o.e[0] = e0; o.e[1] = e1; o.e[2] = e2; o.e[3] = e3;
    return o;
}

/* Spilled error bounds are stored as four bf16 rounded towards +inf: a bound
   needs range, not precision, and rounding up keeps it a bound. */
__device__ __forceinline__ uint2 rc_pack_err(float a, float b, float c, float d)
{
    __nv_bfloat162 lo = __halves2bfloat162(__float2bfloat16_ru(a), __float2bfloat16_ru(b));
    __nv_bfloat162 hi = __halves2bfloat162(__float2bfloat16_ru(c), __float2bfloat16_ru(d));
    uint2 u;
    u.x = *reinterpret_cast<unsigned int *>(&lo);
    u.y = *reinterpret_cast<unsigned int *>(&hi);
    return u;
}

__device__ __forceinline__ float4 rc_unpack_err(uint2 u)
{
    __nv_bfloat162 lo = *reinterpret_cast<__nv_bfloat162 *>(&u.x);
    __nv_bfloat162 hi = *reinterpret_cast<__nv_bfloat162 *>(&u.y);
    const float2 a = __bfloat1622float2(lo), b = __bfloat1622float2(hi);
    return make_float4(a.x, a.y, b.x, b.y);
}

/* Evaluate one decoded program on this thread's four rows starting at
   `myrow`. Features come from the staged shared tile `xs` ([k][T] float4)
   when `staged`, else straight from global memory. `stk`/`estk` are the
   spill slots ([slot][T]). Returns predictions p and error bounds pe. */
template <int T, bool TRACK>
__device__ __forceinline__ void rc_run(const RcIns *__restrict__ prog, const float4 *xs,
                                       bool staged, const float *__restrict__ cols, int npad,
                                       int myrow, float4 *stk, uint2 *estk, int tid, float4 &p,
                                       float4 &pe)
{
    float t0 = 0.f, t1 = 0.f, t2 = 0.f, t3 = 0.f;
    float e0 = 0.f, e1 = 0.f, e2 = 0.f, e3 = 0.f;
    for (int pc = 0; pc < RC_MAX_INS; ++pc) {
        const RcIns in = prog[pc];
        const unsigned kind = in.kind;
        if (kind <= K_PUSH_CONST) {
            if (in.spill != 0xff) {
                stk[in.spill * T + tid] = make_float4(t0, t1, t2, t3);
                if (TRACK) estk[in.spill * T + tid] = rc_pack_err(e0, e1, e2, e3);
            }
            if (kind == K_PUSH_VAR) {
                const float4 x = staged ? xs[in.imm * T + tid]
                                        : __ldg(reinterpret_cast<const float4 *>(
                                              cols + (size_t)in.imm * (size_t)npad + myrow));
                t0 = x.x; t1 = x.y; t2 = x.z; t3 = x.w;
            } else {
                const float c = __uint_as_float(in.imm);
                t0 = c; t1 = c; t2 = c; t3 = c;
            }
            e0 = e1 = e2 = e3 = 0.0f;
            continue;
        }
        if (kind == K_UNARY) {
            switch (in.op) {
                case OP_SIN: RC_U4(OP_SIN); break;
                case OP_COS: RC_U4(OP_COS); break;
                case OP_EXP: RC_U4(OP_EXP); break;
                case OP_LOG: RC_U4(OP_LOG); break;
                case OP_SQRT: RC_U4(OP_SQRT); break;
                case OP_SQUARE: RC_U4(OP_SQUARE); break;
                case OP_NEG: RC_U4(OP_NEG); break;
                default: {
                    RcF8 v;
                    v.t[0] = t0; v.t[1] = t1; v.t[2] = t2; v.t[3] = t3;
                    v.e[0] = e0; v.e[1] = e1; v.e[2] = e2; v.e[3] = e3;
                    const RcF8 o = rc_un4_rare<TRACK>(in.op, v);
                    t0 = o.t[0]; t1 = o.t[1]; t2 = o.t[2]; t3 = o.t[3];
                    e0 = o.e[0]; e1 = o.e[1]; e2 = o.e[2]; e3 = o.e[3];
                } break;
            }
            continue;
        }
        if (kind <= K_BIN_C) {
            float a0, a1, a2, a3, b0, b1, b2, b3;
            float ea0 = 0.f, ea1 = 0.f, ea2 = 0.f, ea3 = 0.f;
            float eb0 = 0.f, eb1 = 0.f, eb2 = 0.f, eb3 = 0.f;
            if (kind == K_BIN_S) {
                const float4 a = stk[in.arg * T + tid];
                a0 = a.x; a1 = a.y; a2 = a.z; a3 = a.w;
                b0 = t0; b1 = t1; b2 = t2; b3 = t3;
                if (TRACK) {
                    const float4 ea = rc_unpack_err(estk[in.arg * T + tid]);
                    ea0 = ea.x; ea1 = ea.y; ea2 = ea.z; ea3 = ea.w;
                    eb0 = e0; eb1 = e1; eb2 = e2; eb3 = e3;
                }
            } else {
                a0 = t0; a1 = t1; a2 = t2; a3 = t3;
                ea0 = e0; ea1 = e1; ea2 = e2; ea3 = e3;
                if (kind == K_BIN_V) {
                    const float4 b = staged ? xs[in.imm * T + tid]
                                            : __ldg(reinterpret_cast<const float4 *>(
                                                  cols + (size_t)in.imm * (size_t)npad + myrow));
                    b0 = b.x; b1 = b.y; b2 = b.z; b3 = b.w;
                } else {
                    const float c = __uint_as_float(in.imm);
                    b0 = c; b1 = c; b2 = c; b3 = c;
                }
            }
            switch (in.op) {
                case OP_ADD: RC_B4(OP_ADD); break;
                case OP_SUB: RC_B4(OP_SUB); break;
                case OP_MUL: RC_B4(OP_MUL); break;
                case OP_DIV: RC_B4(OP_DIV); break;
                case OP_POW: RC_B4(OP_POW); break;
                default: {
                    RcB16 v;
                    v.a[0] = a0; v.a[1] = a1; v.a[2] = a2; v.a[3] = a3;
                    v.b[0] = b0; v.b[1] = b1; v.b[2] = b2; v.b[3] = b3;
                    v.ea[0] = ea0; v.ea[1] = ea1; v.ea[2] = ea2; v.ea[3] = ea3;
                    v.eb[0] = eb0; v.eb[1] = eb1; v.eb[2] = eb2; v.eb[3] = eb3;
                    const RcF8 o = rc_bin4_rare<TRACK>(in.op, v);
                    t0 = o.t[0]; t1 = o.t[1]; t2 = o.t[2]; t3 = o.t[3];
                    e0 = o.e[0]; e1 = o.e[1]; e2 = o.e[2]; e3 = o.e[3];
                } break;
            }
            continue;
        }
        if (kind == K_IF) {
            /* Both arms are evaluated; the select discards the other one, NaN
               included (eval.cu:515-521). */
            const float4 cnd = stk[in.arg * T + tid];
            const float4 a = stk[(in.arg + 1) * T + tid];
            if (TRACK) {
                const float4 ec = rc_unpack_err(estk[in.arg * T + tid]);
                const float4 ea = rc_unpack_err(estk[(in.arg + 1) * T + tid]);
                e0 = (ec.x > 0.f && fabsf(cnd.x) <= ec.x) ? fabsf(a.x - t0) + fmaxf(ea.x, e0)
                                                          : (cnd.x > 0.f ? ea.x : e0);
                e1 = (ec.y > 0.f && fabsf(cnd.y) <= ec.y) ? fabsf(a.y - t1) + fmaxf(ea.y, e1)
                                                          : (cnd.y > 0.f ? ea.y : e1);
                e2 = (ec.z > 0.f && fabsf(cnd.z) <= ec.z) ? fabsf(a.z - t2) + fmaxf(ea.z, e2)
                                                          : (cnd.z > 0.f ? ea.z : e2);
                e3 = (ec.w > 0.f && fabsf(cnd.w) <= ec.w) ? fabsf(a.w - t3) + fmaxf(ea.w, e3)
                                                          : (cnd.w > 0.f ? ea.w : e3);
            }
            t0 = cnd.x > 0.0f ? a.x : t0;
            t1 = cnd.y > 0.0f ? a.y : t1;
            t2 = cnd.z > 0.0f ? a.z : t2;
            t3 = cnd.w > 0.0f ? a.w : t3;
            continue;
        }
        if (kind == K_HALT) {
            if (in.arg == 1) {
                p = make_float4(t0, t1, t2, t3);
                pe = make_float4(e0, e1, e2, e3);
            } else {
                /* the reference returns s[0] (eval.cu:429) */
                p = stk[tid];
                pe = TRACK ? rc_unpack_err(estk[tid]) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
            return;
        }
        break; /* K_NAN */
    }
    p = make_float4(rc_nanf(), rc_nanf(), rc_nanf(), rc_nanf());
    pe = make_float4(0.f, 0.f, 0.f, 0.f);
}

/* The f32 row loss of the legacy evaluator (eval.cu:712-727). */
__device__ __forceinline__ float rc_row_loss(float r, int loss)
{
    if (loss == 1) {
        const float rr = r * r;
        return isfinite(rr) ? log1pf(rr) : 2.0f * logf(fabsf(r));
    }
    if (loss == 4) return fabsf(r);
    if (loss != 0) return rc_nanf();
    return r * r;
}

__device__ __forceinline__ double rc_sigmoid_d(double x)
{
    if (x >= 0.0) return 1.0 / (1.0 + exp(-x));
    const double e = exp(x);
    return e / (1.0 + e);
}

/* Labelled row loss (eval.cu:696-728 `rc_class_row_loss`, metrics.rs
   `classification_row_loss`), evaluated in f64 on the (f32) prediction. */
__device__ __forceinline__ double rc_class_row_loss_d(double p, double tsign, int loss)
{
    const double u = tsign * p;
    if (loss == SM_LOG_LOSS) {
        const double a = fabs(u);
        return (u < 0.0 ? -u : 0.0) + log1p(exp(-a));
    }
    if (loss == SM_BRIER) {
        const double l = 0.5 * (tsign + 1.0);
        const double d = rc_sigmoid_d(p) - l;
        return d * d;
    }
    if (loss == SM_HINGE_ORDINARY) {
        const double h = 1.0 - u;
        return h > 0.0 ? h : 0.0;
    }
    if (loss == SM_HINGE_SQUARED) {
        const double h = 1.0 - u;
        return h > 0.0 ? h * h : 0.0;
    }
    if (loss == SM_HINGE_SIGMOID) {
        const double s = 2.0 * rc_sigmoid_d(p) - 1.0;
        const double h = 1.0 - tsign * s;
        return h > 0.0 ? h : 0.0;
    }
    return CUDART_NAN;
}

struct ScoreArgs {
    const float *cols;
    const float *y;
    const float *tsign;
    const double *w;
    int n, npad, v;
    int staged;
    const RcIns *ins;
    const int *ins_off;
    const int *ins_len;   /* [P] instructions per program, or null: ins_off[p + 1] - ins_off[p] */
    const int *order;     /* candidate ids of this bucket, longest first */
    int ncand;            /* candidates in this bucket */
    int group;            /* candidates per work item */
    int subtiles;         /* sub-tiles (T*4 rows each) per tile */
    int ntiles;
    int nitems;
    int maxins;
    int nslots;
    int *counter;
    double *part;         /* [4][P][ptiles]: a0, a1, e0, e1 */
    int nprog;
    int ptiles;
    int *bad;             /* [P] */
    int *badrow;          /* [P] or null: first 4-row group of a hard failure */
    unsigned long long *rows; /* or null: [0] += rows the interpreter evaluated,
                                 [2] += those rows x (ops + 2) of their candidate */
    const int *opw;           /* [P] postfix ops + 2 per candidate (with rows) */
    float *pred;          /* SM_PREDICT: [P][n] */
    const double *pbar;   /* SM_CORR_PASS2: per-candidate mean prediction */
    const double *pbar_err;
    double ybar;
    int mode;
};

/* Per-row accumulation of one candidate: a0/a1 the objective's sums, e0/e1
   their error bounds. Returns without touching them for a hard-failure row
   (which sets `bad`). */
__device__ __forceinline__ void rc_accumulate(const ScoreArgs &a, int mode, float pr, float pe,
                                              float yv, int row, int cand, double &a0,
                                              double &a1, double &e0, double &e1, int &bad)
{
    const bool finite = isfinite(pr) && fabsf(pr) <= 1e30f;
    if (mode >= SM_EVAL_SQUARED && mode <= SM_EVAL_ABSOLUTE) {
        if (!finite) a0 += 1e30;
        else a0 += (double)rc_row_loss(pr - yv, mode - SM_EVAL_SQUARED);
        return;
    }
    if (mode == SM_PREDICT) {
        a.pred[(size_t)cand * (size_t)a.n + (size_t)row] = pr;
        return;
    }
    const double E = (double)pe;
    if (mode >= SM_LOG_LOSS && mode <= SM_HINGE_SQUARED) {
        const double wi = a.w ? a.w[row] : 1.0;
        if (!isfinite(wi) || wi < 0.0) {
            bad = 1;
            return;
        }
        if (wi == 0.0) return;
        const float t = a.tsign ? a.tsign[row] : rc_nanf();
        if (!isfinite(t) || !finite) {
            bad = 1;
            return;
        }
        a0 += wi * rc_class_row_loss_d((double)pr, (double)t, mode);
        a1 += wi;
        const double h = fabs(1.0 - (double)t * (double)pr);
        e0 += wi * E * (1.0 + 2.0 * (h + E));
        return;
    }
    if (!finite) {
        bad = 1;
        return;
    }
    if (mode == SM_CORR_PASS1) {
        a0 += (double)pr;
        e0 += E;
        return;
    }
    if (mode == SM_CORR_PASS2) {
        const double dp = (double)pr - a.pbar[cand];
        const double dy = (double)yv - a.ybar;
        const double Et = E + a.pbar_err[cand];
        a0 += dp * dp;
        a1 += dp * dy;
        e0 += (2.0 * fabs(dp) + Et) * Et;
        e1 += fabs(dy) * Et;
        return;
    }
    const double r = (double)pr - (double)yv;
    switch (mode) {
        case SM_ABSOLUTE:
            a0 += fabs(r);
            e0 += E;
            break;
        case SM_LOG_SQUASHED: {
            const double rr = r * r;
            a0 += isfinite(rr) ? log1p(rr) : 2.0 * log(fabs(r));
            const double lo = fmax(fabs(r) - E, 0.0);
            e0 += (2.0 * fabs(r) + E) * E / (1.0 + lo * lo);
        } break;
        case SM_SIGNED:
            a0 += r;
            e0 += E;
            break;
        case SM_MAXIMUM:
            a0 = fmax(a0, fabs(r));
            e0 = fmax(e0, E);
            break;
        default:
            a0 += r * r;
            e0 += (2.0 * fabs(r) + E) * E;
            break;
    }
}

/* Butterfly sum over the warp: the same fixed order in every lane. */
__device__ __forceinline__ double rc_warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double rc_warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

/* Shared layout of the f32 scoring kernel. */
template <int T>
struct ScoreSmem {
    static __host__ __device__ size_t xs_bytes(int v, int staged) { return staged ? (size_t)v * T * 16 : 0; }
    static __host__ __device__ size_t stk_bytes(int nslots) { return (size_t)nslots * T * 24; }
    static __host__ __device__ size_t warp_bytes(int group) { return (size_t)group * (T / 32) * 4 * 8; }
    static __host__ __device__ size_t prog_bytes(int group, int maxins) { return (size_t)group * maxins * sizeof(RcIns); }
    static __host__ __device__ size_t total(int v, int staged, int nslots, int group, int maxins)
    {
        return xs_bytes(v, staged) + stk_bytes(nslots) + warp_bytes(group) + prog_bytes(group, maxins);
    }
};

template <int T, bool TRACK>
__global__ void __launch_bounds__(T) rc_score_kernel(ScoreArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NW = T / 32;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    float4 *stk = reinterpret_cast<float4 *>(smem_raw + ScoreSmem<T>::xs_bytes(a.v, a.staged));
    uint2 *estk = reinterpret_cast<uint2 *>(stk + a.nslots * T);
    double *swarp = reinterpret_cast<double *>(estk + a.nslots * T);
    RcIns *sprog = reinterpret_cast<RcIns *>(swarp + a.group * NW * 4);
    __shared__ int s_item;
    __shared__ unsigned s_bad;
    __shared__ unsigned long long s_rows, s_ops;
    const int SUB = T * 4;
    const int mode = a.mode;
    const bool skip_bad = rc_mode_tracks(mode);

    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= a.nitems) break;
        const int g = item / a.ntiles;
        const int tile = item - g * a.ntiles;
        const int cbase = g * a.group;
        const int gcount = min(a.group, a.ncand - cbase);

        unsigned skipmask = 0;
        for (int c = 0; c < gcount; ++c) {
            const int cand = a.order[cbase + c];
            const int b = a.ins_off[cand];
            const int e = a.ins_len ? b + a.ins_len[cand] : a.ins_off[cand + 1];
            for (int q = tid; q < e - b; q += T) sprog[c * a.maxins + q] = a.ins[b + q];
            if (skip_bad && *((volatile int *)(a.bad + cand))) skipmask |= 1u << c;
        }
        for (int q = tid; q < gcount * NW * 4; q += T) swarp[q] = 0.0;
        if (tid == 0) {
            s_bad = 0;
            s_rows = 0;
            s_ops = 0;
        }
        __syncthreads();

        /* each warp runs one candidate over all of the tile's rows before its
           single reduction; the features come straight from L2 */
        for (int c = 0; c < gcount; ++c) {
            /* a candidate already known to be a hard failure skips its rows */
            if (skip_bad && (skipmask & (1u << c))) continue;
            const int cand = a.order[cbase + c];
            double a0 = 0.0, a1 = 0.0, e0 = 0.0, e1 = 0.0;
            int bad = 0;
            int wrows = 0; /* rows of this warp the candidate was evaluated on */
            for (int s = 0; s < a.subtiles; ++s) {
                const int row0 = (tile * a.subtiles + s) * SUB;
                if (row0 >= a.n) break;
                const int myrow = row0 + 4 * tid;
                wrows += max(0, min(128, a.n - (row0 + 128 * warp)));
                float4 p, pe;
                rc_run<T, TRACK>(sprog + c * a.maxins, nullptr, false, a.cols, a.npad, myrow, stk,
                                 estk, tid, p, pe);
                const float4 yv4 = __ldg(reinterpret_cast<const float4 *>(a.y + myrow));
                const float pr[4] = {p.x, p.y, p.z, p.w};
                const float pq[4] = {pe.x, pe.y, pe.z, pe.w};
                const float yy[4] = {yv4.x, yv4.y, yv4.z, yv4.w};
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int row = myrow + i;
                    if (row < a.n)
                        rc_accumulate(a, mode, pr[i], pq[i], yy[i], row, cand, a0, a1, e0, e1,
                                      bad);
                }
                /* a hard failure ends this warp's rows of the candidate; the
                   lowest failing 4-row group is kept for the f64 re-check */
                if (skip_bad && __any_sync(0xffffffffu, bad)) {
                    const int grp = __reduce_min_sync(0xffffffffu,
                                                      bad ? (unsigned)myrow : 0x7fffffffu);
                    if (a.badrow && lane == 0) atomicMin(a.badrow + cand, grp);
                    break;
                }
            }
            if (a.rows && lane == 0 && wrows > 0) {
                atomicAdd(&s_rows, (unsigned long long)wrows);
                atomicAdd(&s_ops, (unsigned long long)wrows * (unsigned long long)a.opw[cand]);
            }
            if (mode == SM_PREDICT) continue;
            if (mode == SM_MAXIMUM) {
                a0 = rc_warp_max(a0);
                e0 = rc_warp_max(e0);
            } else {
                a0 = rc_warp_sum(a0);
                if (TRACK) e0 = rc_warp_sum(e0);
                if (mode == SM_CORR_PASS2 || (mode >= SM_LOG_LOSS && mode <= SM_HINGE_SQUARED)) {
                    a1 = rc_warp_sum(a1);
                    if (TRACK) e1 = rc_warp_sum(e1);
                }
            }
            const unsigned anybad = __any_sync(0xffffffffu, bad);
            if (lane == 0) {
                double *sw = swarp + (c * NW + warp) * 4;
                sw[0] = a0;
                sw[1] = a1;
                sw[2] = e0;
                sw[3] = e1;
                if (anybad) atomicOr(&s_bad, 1u << c);
            }
        }
        __syncthreads();

        /* Warps in ascending order: one partial per (candidate, tile). */
        if (tid < gcount * 4 && mode != SM_PREDICT) {
            const int c = tid >> 2, q = tid & 3;
            const int cand = a.order[cbase + c];
            double s = 0.0;
            for (int w = 0; w < NW; ++w) {
                const double v = swarp[(c * NW + w) * 4 + q];
                s = (mode == SM_MAXIMUM) ? fmax(s, v) : s + v;
            }
            a.part[((size_t)q * a.nprog + cand) * a.ptiles + tile] = s;
            if (q == 0 && (s_bad & (1u << c)) && !(skipmask & (1u << c))) atomicOr(&a.bad[cand], 1);
        }
        if (a.rows && tid == 0 && s_rows) {
            atomicAdd(a.rows, s_rows);
            atomicAdd(a.rows + 2, s_ops);
        }
        __syncthreads();
    }
}

/* Tiles of each candidate in ascending order: the final, fixed-order sums,
   the objective, the status, and the flag that sends the candidate to the
   f64 lane (a non-finite f32 row, or an error bound above RC_FLAG_TOL of the
   objective's sums). */
__global__ void rc_score_finalize(int nprog, const int *__restrict__ cand_tiles,
                                  const double *__restrict__ part, int ptiles,
                                  const int *__restrict__ bad, int n, int mode, double syy,
                                  double *__restrict__ out, int *__restrict__ status,
                                  float *__restrict__ out_f32, double *__restrict__ pbar,
                                  double *__restrict__ pbar_err, int *__restrict__ nflag,
                                  int *__restrict__ flagged)
{
    const int cand = blockIdx.x * blockDim.x + threadIdx.x;
    if (cand >= nprog) return;
    const int nt = cand_tiles[cand];
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int q = 0; q < 4; ++q) {
        for (int t = 0; t < nt; ++t) {
            const double v = part[((size_t)q * nprog + cand) * ptiles + t];
            s[q] = (mode == SM_MAXIMUM) ? fmax(s[q], v) : s[q] + v;
        }
    }
    if (mode >= SM_EVAL_SQUARED && mode <= SM_EVAL_ABSOLUTE) {
        out_f32[cand] = (float)s[0];
        return;
    }
    if (mode == SM_PREDICT) return;
    const double dn = (double)n;
    /* (the comparisons below flag a bound that is not a number) */
    bool flag = false;
    if (bad[cand]) {
        if (out) out[cand] = INFINITY;
        if (status) status[cand] = RC_SCORE_NONFINITE;
        flag = true;
    } else if (mode == SM_CORR_PASS1) {
        pbar[cand] = s[0] / dn;
        pbar_err[cand] = s[2] / dn;
        return;
    } else {
        double v = 0.0;
        int st = 0;
        switch (mode) {
            case SM_CORRELATION:
            case SM_CORRELATION_SIGNED: {
                /* s0 = sum dp^2, s1 = sum dp dy; the CPU rule: zero variance
                   on either side is rho = 0 (eval.cu:1003-1012). */
                const double rho = (s[0] <= 0.0 || syy <= 0.0) ? 0.0
                                                               : s[1] / (sqrt(s[0]) * sqrt(syy));
                v = mode == SM_CORRELATION_SIGNED ? 1.0 - rho : 1.0 - fabs(rho);
                flag = !(s[2] <= RC_FLAG_TOL * s[0]) ||
                       !(s[3] <= RC_FLAG_TOL * (fabs(s[1]) + RC_FLAG_TOL * sqrt(fmax(s[0], 0.0) * syy)));
            } break;
            case SM_AIC: case SM_AICC: case SM_BIC:
                v = s[0]; /* RSS; the host applies the penalty */
                flag = !(s[2] <= RC_FLAG_TOL * fabs(s[0]));
                break;
            case SM_SIGNED:
                v = fabs(s[0]) / dn;
                flag = !(s[2] <= RC_FLAG_TOL * fabs(s[0]));
                break;
            case SM_MAXIMUM:
                v = s[0];
                flag = !(s[2] <= RC_FLAG_TOL * s[0]);
                break;
            case SM_LOG_LOSS: case SM_BRIER: case SM_HINGE_SIGMOID: case SM_HINGE_ORDINARY:
            case SM_HINGE_SQUARED:
                if (!(s[1] > 0.0)) {
                    v = INFINITY;
                    st = RC_SCORE_ALL_ZERO_WEIGHT;
                } else {
                    v = s[0] / s[1];
                    flag = !(s[2] <= RC_FLAG_TOL * fabs(s[0]));
                }
                break;
            default:
                v = s[0] / dn;
                flag = !(s[2] <= RC_FLAG_TOL * fabs(s[0]));
                break;
        }
        out[cand] = v;
        status[cand] = st;
    }
    if (mode == SM_CORR_PASS1) return;
    if (flag && flagged) {
        const int k = atomicAdd(nflag, 1);
        flagged[k] = cand;
    }
}

/* ---- the f64 re-check lane ---------------------------------------------- */

/* expr::eval semantics in f64 (expr.rs:1054-1326) for one unary operator. */
__device__ __forceinline__ double rc_unary_d(unsigned op, double a)
{
    switch (op) {
        case OP_SIN: return sin(a);
        case OP_COS: return cos(a);
        case OP_TAN: {
            const double t = tan(a);
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
        case OP_STEP: return a > 0.0 ? 1.0 : 0.0;
        case OP_SINH: return sinh(a);
        case OP_COSH: return cosh(a);
        case OP_FLOOR: return floor(a);
        case OP_CEIL: return ceil(a);
        case OP_ROUND: return round(a);
        case OP_ERF: return a == 0.0 ? 0.0 : erf(a);
        case OP_ERFC: return erfc(a);
        case OP_SIGN:
            return isnan(a) ? CUDART_NAN : (a > 0.0 ? 1.0 : (a < 0.0 ? -1.0 : 0.0));
        case OP_NOT: return isnan(a) ? CUDART_NAN : (a > 0.0 ? 0.0 : 1.0);
        default: return CUDART_NAN;
    }
}

__device__ __forceinline__ double rc_binary_d(unsigned op, double a, double b)
{
    switch (op) {
        case OP_ADD: return a + b;
        case OP_SUB: return a - b;
        case OP_MUL: return a * b;
        case OP_DIV: return fabs(b) < 1e-12 ? CUDART_NAN : a / b;
        case OP_POW:
            return (a < 0.0 && fabs(b - round(b)) > 1e-9) ? CUDART_NAN : pow(a, b);
        case OP_MOD:
            if (!isfinite(a) || !isfinite(b) || fabs(b) < 1e-12) return CUDART_NAN;
            return a - b * floor(a / b);
        case OP_ATAN2: return (isnan(a) || isnan(b)) ? CUDART_NAN : atan2(a, b);
        case OP_MIN: return (isnan(a) || isnan(b)) ? CUDART_NAN : fmin(a, b);
        case OP_MAX: return (isnan(a) || isnan(b)) ? CUDART_NAN : fmax(a, b);
        case OP_EQUAL: return (isnan(a) || isnan(b)) ? CUDART_NAN : (a == b ? 1.0 : 0.0);
        case OP_LESS: return (isnan(a) || isnan(b)) ? CUDART_NAN : (a < b ? 1.0 : 0.0);
        case OP_LESS_OR_EQUAL:
            return (isnan(a) || isnan(b)) ? CUDART_NAN : (a <= b ? 1.0 : 0.0);
        case OP_GREATER: return (isnan(a) || isnan(b)) ? CUDART_NAN : (a > b ? 1.0 : 0.0);
        case OP_GREATER_OR_EQUAL:
            return (isnan(a) || isnan(b)) ? CUDART_NAN : (a >= b ? 1.0 : 0.0);
        case OP_AND:
            return (isnan(a) || isnan(b)) ? CUDART_NAN : ((a > 0.0 && b > 0.0) ? 1.0 : 0.0);
        case OP_OR:
            return (isnan(a) || isnan(b)) ? CUDART_NAN : ((a > 0.0 || b > 0.0) ? 1.0 : 0.0);
        case OP_XOR:
            return (isnan(a) || isnan(b)) ? CUDART_NAN : (((a > 0.0) != (b > 0.0)) ? 1.0 : 0.0);
        default: return CUDART_NAN;
    }
}

/* f64 evaluation of one decoded program on two rows (the f32 inputs and f32
   constants widened, as the CPU oracle sees them). */
template <int T>
__device__ __forceinline__ double2 rc_run_d(const RcIns *__restrict__ prog,
                                            const float *__restrict__ cols, int npad, int row,
                                            double2 *stk, int tid)
{
    double t0 = 0.0, t1 = 0.0;
    for (int pc = 0; pc < RC_MAX_INS; ++pc) {
        const RcIns in = prog[pc];
        const unsigned kind = in.kind;
        if (kind <= K_PUSH_CONST) {
            if (in.spill != 0xff) stk[in.spill * T + tid] = make_double2(t0, t1);
            if (kind == K_PUSH_VAR) {
                const float2 x = __ldg(reinterpret_cast<const float2 *>(
                    cols + (size_t)in.imm * (size_t)npad + row));
                t0 = x.x;
                t1 = x.y;
            } else {
                t0 = t1 = (double)__uint_as_float(in.imm);
            }
            continue;
        }
        if (kind == K_UNARY) {
            t0 = rc_unary_d(in.op, t0);
            t1 = rc_unary_d(in.op, t1);
            continue;
        }
        if (kind <= K_BIN_C) {
            double a0, a1, b0, b1;
            if (kind == K_BIN_S) {
                const double2 a = stk[in.arg * T + tid];
                a0 = a.x;
                a1 = a.y;
                b0 = t0;
                b1 = t1;
            } else {
                a0 = t0;
                a1 = t1;
                if (kind == K_BIN_V) {
                    const float2 x = __ldg(reinterpret_cast<const float2 *>(
                        cols + (size_t)in.imm * (size_t)npad + row));
                    b0 = x.x;
                    b1 = x.y;
                } else {
                    b0 = b1 = (double)__uint_as_float(in.imm);
                }
            }
            t0 = rc_binary_d(in.op, a0, b0);
            t1 = rc_binary_d(in.op, a1, b1);
            continue;
        }
        if (kind == K_IF) {
            const double2 cnd = stk[in.arg * T + tid];
            const double2 a = stk[(in.arg + 1) * T + tid];
            t0 = cnd.x > 0.0 ? a.x : t0;
            t1 = cnd.y > 0.0 ? a.y : t1;
            continue;
        }
        if (kind == K_HALT) return in.arg == 1 ? make_double2(t0, t1) : stk[tid];
        break;
    }
    return make_double2(CUDART_NAN, CUDART_NAN);
}

struct Score64Args {
    const float *cols;
    const float *y;
    const float *tsign;
    const double *w;
    int n, npad;
    const RcIns *ins;
    const int *ins_off;
    const int *flagged;
    const int *nflag;
    int ntiles;
    int nslots;
    int *counter;
    double *part;      /* [2][P][ptiles] */
    int nprog;
    int ptiles;
    int *bad;          /* [P] */
    const double *pbar;
    double ybar;
    int mode;
    unsigned long long *rows; /* or null: [0] += rows the f64 lane evaluated,
                                 [2] += those rows x (ops + 2) */
    const int *opw;
};

template <int T>
__global__ void __launch_bounds__(T) rc_score64_kernel(Score64Args a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *stk = reinterpret_cast<double2 *>(smem_raw);
    RcIns *sprog = reinterpret_cast<RcIns *>(stk + a.nslots * T);
    double *red = reinterpret_cast<double *>(sprog + RC_MAX_INS);
    __shared__ int s_item, s_known;
    const int tid = threadIdx.x;
    const int SUB = 2 * T;
    const int subtiles = RC_TILE_ROWS / SUB;
    const int mode = a.mode;
    for (;;) {
        const int total = *a.nflag * a.ntiles;
        if (tid == 0) {
            s_item = atomicAdd(a.counter, 1);
            s_known = s_item < total ? *((volatile int *)(a.bad + a.flagged[s_item / a.ntiles]))
                                     : 0;
        }
        __syncthreads();
        const int item = s_item;
        if (item >= total) break;
        /* a candidate already shown non-finite needs no more rows (its
           partial sums are not read) */
        if (s_known) {
            __syncthreads();
            continue;
        }
        const int cand = a.flagged[item / a.ntiles];
        const int tile = item % a.ntiles;
        const int b = a.ins_off[cand], e = a.ins_off[cand + 1];
        for (int q = tid; q < e - b; q += T) sprog[q] = a.ins[b + q];
        __syncthreads();
        double a0 = 0.0, a1 = 0.0;
        int bad = 0;
        int trows = 0;
        for (int s = 0; s < subtiles; ++s) {
            const int row0 = (tile * subtiles + s) * SUB;
            if (row0 >= a.n) break;
            if (*((volatile int *)(a.bad + cand))) break;
            trows += min(SUB, a.n - row0);
            const int myrow = row0 + 2 * tid;
            const double2 p = rc_run_d<T>(sprog, a.cols, a.npad, myrow, stk, tid);
            const double pr[2] = {p.x, p.y};
            for (int i = 0; i < 2; ++i) {
                const int row = myrow + i;
                if (row >= a.n) continue;
                const double yv = (double)a.y[row];
                const double v = pr[i];
                if (mode >= SM_LOG_LOSS && mode <= SM_HINGE_SQUARED) {
                    const double wi = a.w ? a.w[row] : 1.0;
                    if (!isfinite(wi) || wi < 0.0) { bad = 1; continue; }
                    if (wi == 0.0) continue;
                    const double t = a.tsign ? (double)a.tsign[row] : CUDART_NAN;
                    if (!isfinite(t) || !isfinite(v) || fabs(v) > 1e30) { bad = 1; continue; }
                    a0 += wi * rc_class_row_loss_d(v, t, mode);
                    a1 += wi;
                    continue;
                }
                if (!isfinite(v) || fabs(v) > 1e30) {
                    bad = 1;
                    continue;
                }
                if (mode == SM_CORR_PASS1) { a0 += v; continue; }
                if (mode == SM_CORR_PASS2) {
                    const double dp = v - a.pbar[cand];
                    a0 += dp * dp;
                    a1 += dp * (yv - a.ybar);
                    continue;
                }
                const double r = v - yv;
                switch (mode) {
                    case SM_ABSOLUTE: a0 += fabs(r); break;
                    case SM_LOG_SQUASHED: {
                        const double rr = r * r;
                        a0 += isfinite(rr) ? log1p(rr) : 2.0 * log(fabs(r));
                    } break;
                    case SM_SIGNED: a0 += r; break;
                    case SM_MAXIMUM: a0 = fmax(a0, fabs(r)); break;
                    default: a0 += r * r; break;
                }
            }
            if (bad) atomicOr(a.bad + cand, 1);
        }
        if (a.rows && tid == 0 && trows > 0) {
            atomicAdd(a.rows, (unsigned long long)trows);
            atomicAdd(a.rows + 2, (unsigned long long)trows * (unsigned long long)a.opw[cand]);
        }
        /* fixed-order block trees */
        for (int q = 0; q < 2; ++q) {
            red[tid] = q == 0 ? a0 : a1;
            __syncthreads();
            for (int st = T / 2; st > 0; st >>= 1) {
                if (tid < st) red[tid] = mode == SM_MAXIMUM ? fmax(red[tid], red[tid + st])
                                                            : red[tid] + red[tid + st];
                __syncthreads();
            }
            if (tid == 0) a.part[((size_t)q * a.nprog + cand) * a.ptiles + tile] = red[0];
            __syncthreads();
        }
    }
}

/* A row's hard failure in the f64 lane (the rule of rc_score64_kernel): a
   prediction that is not finite or beyond 1e30, and for the classification
   objectives an invalid weight or label. */
__device__ __forceinline__ bool rc_row64_bad(const Score64Args &a, double v, int row)
{
    if (a.mode >= SM_LOG_LOSS && a.mode <= SM_HINGE_SQUARED) {
        const double wi = a.w ? a.w[row] : 1.0;
        if (!isfinite(wi) || wi < 0.0) return true;
        if (wi == 0.0) return false;
        const double t = a.tsign ? (double)a.tsign[row] : CUDART_NAN;
        return !isfinite(t) || !isfinite(v) || fabs(v) > 1e30;
    }
    return !isfinite(v) || fabs(v) > 1e30;
}

/* Before the f64 lane: each flagged candidate that failed in f32 has its
   failing 4-row group evaluated in f64 first (one warp per candidate, two
   lanes with two rows each). A failure there is a failure of the whole
   candidate in f64, exactly what the lane's scan would find, so the lane
   skips it; otherwise the lane scans all rows as before. */
template <int T>
__global__ void __launch_bounds__(T) rc_badrow_check(Score64Args a, const int *badrow)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *stk = reinterpret_cast<double2 *>(smem_raw);
    RcIns *sprog = reinterpret_cast<RcIns *>(stk + a.nslots * T);
    const int k = blockIdx.x, tid = threadIdx.x;
    if (k >= *a.nflag) return;
    const int cand = a.flagged[k];
    const int r = badrow[cand];
    if (r < 0 || r >= a.n) return;
    const int b = a.ins_off[cand], e = a.ins_off[cand + 1];
    for (int q = tid; q < e - b; q += T) sprog[q] = a.ins[b + q];
    __syncthreads();
    if (tid >= 2) return;
    const int myrow = r + 2 * tid;
    const double2 p = rc_run_d<T>(sprog, a.cols, a.npad, myrow, stk, tid);
    const bool b0 = myrow < a.n && rc_row64_bad(a, p.x, myrow);
    const bool b1 = myrow + 1 < a.n && rc_row64_bad(a, p.y, myrow + 1);
    if (b0 || b1) atomicOr(a.bad + cand, 1);
}

/* Overwrite the flagged candidates' results with the f64 lane's. */
__global__ void rc_score64_finalize(const int *__restrict__ flagged, const int *__restrict__ nflag,
                                    int ntiles, const double *__restrict__ part, int nprog,
                                    int ptiles, const int *__restrict__ bad, int n, int mode,
                                    double syy, double *__restrict__ out, int *__restrict__ status,
                                    double *__restrict__ pbar)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= *nflag) return;
    const int cand = flagged[k];
    double s0 = 0.0, s1 = 0.0;
    for (int t = 0; t < ntiles; ++t) {
        const double v0 = part[(size_t)cand * ptiles + t];
        const double v1 = part[((size_t)nprog + cand) * ptiles + t];
        s0 = mode == SM_MAXIMUM ? fmax(s0, v0) : s0 + v0;
        s1 += v1;
    }
    const double dn = (double)n;
    if (mode == SM_CORR_PASS1) {
        pbar[cand] = s0 / dn;
        return;
    }
    if (bad[cand]) {
        out[cand] = INFINITY;
        status[cand] = RC_SCORE_NONFINITE;
        return;
    }
    double v;
    int st = 0;
    switch (mode) {
        case SM_CORRELATION: case SM_CORRELATION_SIGNED: {
            const double rho = (s0 <= 0.0 || syy <= 0.0) ? 0.0 : s1 / (sqrt(s0) * sqrt(syy));
            v = mode == SM_CORRELATION_SIGNED ? 1.0 - rho : 1.0 - fabs(rho);
        } break;
        case SM_AIC: case SM_AICC: case SM_BIC: v = s0; break;
        case SM_SIGNED: v = fabs(s0) / dn; break;
        case SM_MAXIMUM: v = s0; break;
        case SM_LOG_LOSS: case SM_BRIER: case SM_HINGE_SIGMOID: case SM_HINGE_ORDINARY:
        case SM_HINGE_SQUARED:
            if (!(s1 > 0.0)) {
                v = INFINITY;
                st = RC_SCORE_ALL_ZERO_WEIGHT;
            } else {
                v = s0 / s1;
            }
            break;
        default: v = s0 / dn; break;
    }
    out[cand] = v;
    status[cand] = st;
}
