/*
 * Batched scoring of postfix bytecode over the resident rows.
 *
 * Replaces the reference's one-block-per-candidate interpreters
 * (my-version/src/cuda/eval.cu:759-828 `eval_kernel`/`eval_pool_kernel`,
 * :846-1088 `score_kernel<MODE>`, :1093-1104 `predict_kernel`) with one
 * persistent kernel per stack-depth bucket:
 *
 *  - programs are decoded on the host into a top-of-stack-in-registers
 *    instruction stream (rc_decode_postfix); each thread evaluates four
 *    consecutive rows at once, so one warp-uniform dispatch drives four rows
 *    and deeper stack entries live in fixed per-thread shared-memory slots;
 *  - a work item is (a group of G candidates of similar length, a tile of
 *    rows): the tile's feature rows are staged once in shared memory and
 *    reused by all G candidates, which divides the L2 traffic of the feature
 *    matrix by G;
 *  - items are handed out by an atomic counter over groups ordered by
 *    decreasing program length (longest first), so uneven lengths do not
 *    leave a tail;
 *  - every candidate's loss is accumulated in f64 from f32 rows in a fixed
 *    order (per thread, then a fixed block tree per tile, then tiles in
 *    ascending order in the finalize kernel). The tile shape depends only on
 *    the row count and the program's own depth bucket, so a candidate's bits
 *    do not depend on the batch it is scored in.
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "rc_internal.h"
#include "rc_ops.cuh"

/* Internal scoring modes. 0..9 are the RC_SCORE_* regression codes
   (eval.cu:609-619); the rest are internal. */
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

/* ---- host decoder --------------------------------------------------- */

static bool is_binary(uint32_t w)
{
    switch (w) {
        case OP_ADD: case OP_SUB: case OP_MUL: case OP_DIV: case OP_POW: case OP_MOD:
        case OP_ATAN2: case OP_MIN: case OP_MAX: case OP_EQUAL: case OP_LESS:
        case OP_LESS_OR_EQUAL: case OP_GREATER: case OP_GREATER_OR_EQUAL: case OP_AND:
        case OP_OR: case OP_XOR:
            return true;
        default: return false;
    }
}

/* Operators fused with an immediately preceding push (K_BIN_V / K_BIN_C). */
static bool fusable(uint32_t w)
{
    return w == OP_ADD || w == OP_SUB || w == OP_MUL || w == OP_DIV || w == OP_POW;
}

int rc_decode_postfix(const uint32_t *words, size_t nwords, int v, RcIns *out, int *nslots)
{
    /* Walk the words exactly like the reference's device loop (eval.cu:404-573)
       with a symbolic stack depth; any condition under which the reference
       returns NaN for every row makes the program a single K_NAN. */
    std::vector<RcIns> ins;
    ins.reserve(64);
    int depth = 0, maxslot = -1;
    bool ok = true, halted = false;
    size_t i = 0;
    auto spill_slot = [&](int d) -> uint8_t { return d >= 1 ? (uint8_t)(d - 1) : 0xff; };
    while (i < nwords && ok) {
        uint32_t w = words[i++];
        RcIns in;
        memset(&in, 0, sizeof(in));
        in.spill = 0xff;
        if (w == OP_CONST || w == OP_VAR) {
            if (i >= nwords) { ok = false; break; }
            uint32_t a = words[i++];
            if (depth >= RC_MAX_STACK) { ok = false; break; }
            if (w == OP_VAR && (int64_t)a >= (int64_t)v) { ok = false; break; }
            in.kind = (w == OP_CONST) ? K_PUSH_CONST : K_PUSH_VAR;
            in.spill = spill_slot(depth);
            in.imm = a; /* f32 bits of a constant, or the column of a variable */
            if (depth >= 1) maxslot = std::max(maxslot, depth - 1);
            ++depth;
            ins.push_back(in);
        } else if (w == OP_HALT) {
            if (depth < 1) { ok = false; break; }
            in.kind = K_HALT;
            in.arg = depth == 1 ? 1 : 0;
            ins.push_back(in);
            halted = true;
            break;
        } else if (is_binary(w)) {
            if (depth < 2) { ok = false; break; }
            in.kind = K_BIN_S;
            in.op = (uint8_t)w;
            in.arg = (uint8_t)(depth - 2);
            --depth;
            /* Fuse "push x; op" into one instruction: the push's spill slot is
               exactly the slot the operator would pop. */
            if (!ins.empty() && fusable(w)) {
                RcIns &prev = ins.back();
                if ((prev.kind == K_PUSH_VAR || prev.kind == K_PUSH_CONST) && prev.spill != 0xff &&
                    prev.spill == in.arg) {
                    uint8_t kind = prev.kind == K_PUSH_VAR ? K_BIN_V : K_BIN_C;
                    prev.kind = kind;
                    prev.op = (uint8_t)w;
                    prev.spill = 0xff;
                    continue;
                }
            }
            ins.push_back(in);
        } else if (w == OP_IF) {
            if (depth < 3) { ok = false; break; }
            in.kind = K_IF;
            in.arg = (uint8_t)(depth - 3);
            depth -= 2;
            ins.push_back(in);
        } else {
            /* Unary, including unknown codes, which evaluate to NaN
               (eval.cu:567). */
            if (depth < 1) { ok = false; break; }
            in.kind = K_UNARY;
            in.op = (uint8_t)(w > 255 ? 255 : w);
            if (w > 255 || w == OP_HALT) in.op = 254; /* unknown: NaN */
            ins.push_back(in);
        }
    }
    if (!ok || !halted || (int)ins.size() > RC_MAX_INS) {
        RcIns bad;
        memset(&bad, 0, sizeof(bad));
        bad.kind = K_NAN;
        bad.spill = 0xff;
        out[0] = bad;
        *nslots = 0;
        return 1;
    }
    memcpy(out, ins.data(), sizeof(RcIns) * ins.size());
    *nslots = maxslot + 1;
    return (int)ins.size();
}

/* ---- device interpreter --------------------------------------------- */

#define U4(OPC)                                  \
    {                                            \
        t0 = rc_unary_f(OPC, t0);                \
        t1 = rc_unary_f(OPC, t1);                \
        t2 = rc_unary_f(OPC, t2);                \
        t3 = rc_unary_f(OPC, t3);                \
    }
#define B4(OPC)                                  \
    {                                            \
        t0 = rc_binary_f(OPC, a0, b0);           \
        t1 = rc_binary_f(OPC, a1, b1);           \
        t2 = rc_binary_f(OPC, a2, b2);           \
        t3 = rc_binary_f(OPC, a3, b3);           \
    }

/* Evaluate one decoded program on this thread's four rows. `xs` holds the
   staged feature columns ([k][T] float4), `stk` the spill slots ([slot][T]
   float4). Returns the four predictions in p. */
template <int T>
__device__ __forceinline__ void rc_run(const RcIns *__restrict__ prog, const float4 *xs,
                                       float4 *stk, int tid, float4 &p)
{
    float t0 = 0.f, t1 = 0.f, t2 = 0.f, t3 = 0.f;
    for (int pc = 0; pc < RC_MAX_INS; ++pc) {
        const RcIns in = prog[pc];
        const unsigned kind = in.kind;
        if (kind <= K_PUSH_CONST) {
            if (in.spill != 0xff) stk[in.spill * T + tid] = make_float4(t0, t1, t2, t3);
            if (kind == K_PUSH_VAR) {
                const float4 x = xs[in.imm * T + tid];
                t0 = x.x; t1 = x.y; t2 = x.z; t3 = x.w;
            } else {
                const float c = __uint_as_float(in.imm);
                t0 = c; t1 = c; t2 = c; t3 = c;
            }
            continue;
        }
        if (kind == K_UNARY) {
            switch (in.op) {
                case OP_SIN: U4(OP_SIN); break;
                case OP_COS: U4(OP_COS); break;
                case OP_TAN: U4(OP_TAN); break;
                case OP_EXP: U4(OP_EXP); break;
                case OP_LOG: U4(OP_LOG); break;
                case OP_SQRT: U4(OP_SQRT); break;
                case OP_ABS: U4(OP_ABS); break;
                case OP_TANH: U4(OP_TANH); break;
                case OP_SIG: U4(OP_SIG); break;
                case OP_SQUARE: U4(OP_SQUARE); break;
                case OP_CUBE: U4(OP_CUBE); break;
                case OP_NEG: U4(OP_NEG); break;
                case OP_GAUSS: U4(OP_GAUSS); break;
                case OP_STEP: U4(OP_STEP); break;
                case OP_SINH: U4(OP_SINH); break;
                case OP_COSH: U4(OP_COSH); break;
                case OP_FLOOR: U4(OP_FLOOR); break;
                case OP_CEIL: U4(OP_CEIL); break;
                case OP_ROUND: U4(OP_ROUND); break;
                case OP_ERF: U4(OP_ERF); break;
                case OP_ERFC: U4(OP_ERFC); break;
                case OP_SIGN: U4(OP_SIGN); break;
                case OP_NOT: U4(OP_NOT); break;
                default: t0 = t1 = t2 = t3 = rc_nanf(); break;
            }
            continue;
        }
        if (kind <= K_BIN_C) {
            float a0, a1, a2, a3, b0, b1, b2, b3;
            if (kind == K_BIN_S) {
                const float4 a = stk[in.arg * T + tid];
                a0 = a.x; a1 = a.y; a2 = a.z; a3 = a.w;
                b0 = t0; b1 = t1; b2 = t2; b3 = t3;
            } else if (kind == K_BIN_V) {
                const float4 b = xs[in.imm * T + tid];
                a0 = t0; a1 = t1; a2 = t2; a3 = t3;
                b0 = b.x; b1 = b.y; b2 = b.z; b3 = b.w;
            } else {
                const float c = __uint_as_float(in.imm);
                a0 = t0; a1 = t1; a2 = t2; a3 = t3;
                b0 = c; b1 = c; b2 = c; b3 = c;
            }
            switch (in.op) {
                case OP_ADD: B4(OP_ADD); break;
                case OP_SUB: B4(OP_SUB); break;
                case OP_MUL: B4(OP_MUL); break;
                case OP_DIV: B4(OP_DIV); break;
                case OP_POW: B4(OP_POW); break;
                case OP_MOD: B4(OP_MOD); break;
                case OP_ATAN2: B4(OP_ATAN2); break;
                case OP_MIN: B4(OP_MIN); break;
                case OP_MAX: B4(OP_MAX); break;
                case OP_EQUAL: B4(OP_EQUAL); break;
                case OP_LESS: B4(OP_LESS); break;
                case OP_LESS_OR_EQUAL: B4(OP_LESS_OR_EQUAL); break;
                case OP_GREATER: B4(OP_GREATER); break;
                case OP_GREATER_OR_EQUAL: B4(OP_GREATER_OR_EQUAL); break;
                case OP_AND: B4(OP_AND); break;
                case OP_OR: B4(OP_OR); break;
                case OP_XOR: B4(OP_XOR); break;
                default: t0 = t1 = t2 = t3 = rc_nanf(); break;
            }
            continue;
        }
        if (kind == K_IF) {
            /* Both arms are already evaluated; the select discards the other
               one, NaN included (eval.cu:515-521). */
            const float4 cnd = stk[in.arg * T + tid];
            const float4 a = stk[(in.arg + 1) * T + tid];
            t0 = cnd.x > 0.0f ? a.x : t0;
            t1 = cnd.y > 0.0f ? a.y : t1;
            t2 = cnd.z > 0.0f ? a.z : t2;
            t3 = cnd.w > 0.0f ? a.w : t3;
            continue;
        }
        if (kind == K_HALT) {
            if (in.arg == 1) {
                p = make_float4(t0, t1, t2, t3);
            } else {
                p = stk[tid]; /* the reference returns s[0] (eval.cu:429) */
            }
            return;
        }
        break; /* K_NAN */
    }
    p = make_float4(rc_nanf(), rc_nanf(), rc_nanf(), rc_nanf());
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

__device__ __forceinline__ float rc_sigmoid_f(float x)
{
    if (x >= 0.0f) return 1.0f / (1.0f + expf(-x));
    const float e = expf(x);
    return e / (1.0f + e);
}

/* Labelled row loss (eval.cu:696-728 `rc_class_row_loss`). */
__device__ __forceinline__ float rc_class_row_loss(float p, float tsign, int loss)
{
    const float u = tsign * p;
    if (loss == SM_LOG_LOSS) {
        const float a = fabsf(u);
        return (u < 0.0f ? -u : 0.0f) + log1pf(expf(-a));
    }
    if (loss == SM_BRIER) {
        const float l = 0.5f * (tsign + 1.0f);
        const float d = rc_sigmoid_f(p) - l;
        return d * d;
    }
    if (loss == SM_HINGE_ORDINARY) {
        const float h = 1.0f - u;
        return h > 0.0f ? h : 0.0f;
    }
    if (loss == SM_HINGE_SQUARED) {
        const float h = 1.0f - u;
        return h > 0.0f ? h * h : 0.0f;
    }
    if (loss == SM_HINGE_SIGMOID) {
        const float s = 2.0f * rc_sigmoid_f(p) - 1.0f;
        const float h = 1.0f - tsign * s;
        return h > 0.0f ? h : 0.0f;
    }
    return rc_nanf();
}

struct ScoreArgs {
    const float *cols;
    const float *y;
    const float *tsign;
    const double *w;
    int n, npad, v;
    const RcIns *ins;
    const int *ins_off;
    const int *order;     /* candidate ids of this bucket, longest first */
    int ncand;            /* candidates in this bucket */
    int group;            /* candidates per work item */
    int subtiles;         /* sub-tiles (T*4 rows each) per tile */
    int ntiles;
    int nitems;
    int maxins;
    int nslots;
    int *counter;
    double *partial;      /* [P][ptiles] */
    double *partial2;     /* second moment (correlation pass 2, classification weight) */
    int ptiles;
    int *bad;             /* [P] */
    float *pred;          /* SM_PREDICT: [P][n] */
    const double *pbar;   /* SM_CORR_PASS2: per-candidate mean prediction */
    double ybar;
    int mode;
};

/* Per-row accumulation of one candidate. Returns 1 when the row is a hard
   failure for the scoring modes. */
template <int T>
__device__ __forceinline__ void rc_accumulate(const ScoreArgs &a, int mode, float pr, float yv,
                                              int row, int cand, double &acc, double &acc2,
                                              int &bad)
{
    const bool finite = isfinite(pr) && fabsf(pr) <= 1e30f;
    if (mode >= SM_EVAL_SQUARED && mode <= SM_EVAL_ABSOLUTE) {
        if (!finite) acc += 1e30;
        else acc += (double)rc_row_loss(pr - yv, mode - SM_EVAL_SQUARED);
        return;
    }
    if (mode == SM_PREDICT) {
        a.pred[(size_t)cand * (size_t)a.n + (size_t)row] = pr;
        return;
    }
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
        acc += wi * (double)rc_class_row_loss(pr, t, mode);
        acc2 += wi;
        return;
    }
    if (!finite) {
        bad = 1;
        return;
    }
    if (mode == SM_CORR_PASS1) {
        acc += (double)pr;
        return;
    }
    if (mode == SM_CORR_PASS2) {
        const double dp = (double)pr - a.pbar[cand];
        const double dy = (double)yv - a.ybar;
        acc += dp * dp;
        acc2 += dp * dy;
        return;
    }
    const double r = (double)pr - (double)yv;
    switch (mode) {
        case SM_ABSOLUTE: acc += fabs(r); break;
        case SM_LOG_SQUASHED: {
            const double rr = r * r;
            acc += isfinite(rr) ? log1p(rr) : 2.0 * log(fabs(r));
        } break;
        case SM_SIGNED: acc += r; break;
        case SM_MAXIMUM: acc = fmax(acc, fabs(r)); break;
        default: acc += r * r; break;
    }
}

template <int T, bool STAGED>
__global__ void __launch_bounds__(T) rc_score_kernel(ScoreArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const int nx = a.v + 1;                   /* feature columns + y */
    float4 *xs = reinterpret_cast<float4 *>(smem_raw);
    float4 *stk = xs + (STAGED ? nx * T : 0);
    double *sacc = reinterpret_cast<double *>(stk + a.nslots * T);
    double *sacc2 = sacc + a.group * T;
    RcIns *sprog = reinterpret_cast<RcIns *>(sacc2 + a.group * T);
    __shared__ int s_item;
    __shared__ int s_bad;
    const int SUB = T * 4;
    const int mode = a.mode;

    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= a.nitems) break;
        const int g = item / a.ntiles;
        const int tile = item - g * a.ntiles;
        const int cbase = g * a.group;
        const int gcount = min(a.group, a.ncand - cbase);

        for (int c = 0; c < gcount; ++c) {
            const int cand = a.order[cbase + c];
            const int b = a.ins_off[cand], e = a.ins_off[cand + 1];
            for (int q = tid; q < e - b; q += T) sprog[c * a.maxins + q] = a.ins[b + q];
            sacc[c * T + tid] = 0.0;
            sacc2[c * T + tid] = 0.0;
        }
        if (tid == 0) s_bad = 0;
        unsigned badmask = 0;
        __syncthreads();

        for (int s = 0; s < a.subtiles; ++s) {
            const int row0 = (tile * a.subtiles + s) * SUB;
            if (row0 >= a.n) break;
            const int myrow = row0 + 4 * tid;
            const float4 *yp = reinterpret_cast<const float4 *>(a.y + myrow);
            float4 yv4 = __ldg(yp);
            if (STAGED) {
                for (int k = 0; k < a.v; ++k) {
                    xs[k * T + tid] = __ldg(reinterpret_cast<const float4 *>(
                        a.cols + (size_t)k * (size_t)a.npad + (size_t)myrow));
                }
            }
            __syncthreads();
            for (int c = 0; c < gcount; ++c) {
                const int cand = a.order[cbase + c];
                float4 p;
                if (STAGED) {
                    rc_run<T>(sprog + c * a.maxins, xs, stk, tid, p);
                }
                double acc = sacc[c * T + tid];
                double acc2 = sacc2[c * T + tid];
                int bad = 0;
                const float pr[4] = {p.x, p.y, p.z, p.w};
                const float yy[4] = {yv4.x, yv4.y, yv4.z, yv4.w};
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int row = myrow + i;
                    if (row < a.n) rc_accumulate<T>(a, mode, pr[i], yy[i], row, cand, acc, acc2, bad);
                }
                sacc[c * T + tid] = acc;
                sacc2[c * T + tid] = acc2;
                if (bad) badmask |= 1u << c;
            }
            __syncthreads();
        }

        /* Fixed-order block tree per candidate, then one partial per tile. */
        if (badmask) atomicOr(&s_bad, (int)badmask);
        for (int st = T / 2; st > 0; st >>= 1) {
            if (tid < st) {
                for (int c = 0; c < gcount; ++c) {
                    if (mode == SM_MAXIMUM) {
                        sacc[c * T + tid] = fmax(sacc[c * T + tid], sacc[c * T + tid + st]);
                    } else {
                        sacc[c * T + tid] += sacc[c * T + tid + st];
                        sacc2[c * T + tid] += sacc2[c * T + tid + st];
                    }
                }
            }
            __syncthreads();
        }
        if (tid < gcount) {
            const int cand = a.order[cbase + tid];
            a.partial[(size_t)cand * a.ptiles + tile] = sacc[tid * T];
            if (a.partial2) a.partial2[(size_t)cand * a.ptiles + tile] = sacc2[tid * T];
            if (s_bad & (1 << tid)) atomicOr(&a.bad[cand], 1);
        }
        __syncthreads();
    }
}

/* Global-memory variant for wide tables (more columns than the staging
   budget): identical arithmetic, features read straight from L2. */
template <int T>
__device__ __forceinline__ void rc_run_global(const RcIns *__restrict__ prog, const float *cols,
                                              int npad, int myrow, float4 *stk, int tid, float4 &p)
{
    float t0 = 0.f, t1 = 0.f, t2 = 0.f, t3 = 0.f;
    for (int pc = 0; pc < RC_MAX_INS; ++pc) {
        const RcIns in = prog[pc];
        const unsigned kind = in.kind;
        if (kind <= K_PUSH_CONST) {
            if (in.spill != 0xff) stk[in.spill * T + tid] = make_float4(t0, t1, t2, t3);
            if (kind == K_PUSH_VAR) {
                const float4 x = __ldg(reinterpret_cast<const float4 *>(
                    cols + (size_t)in.imm * (size_t)npad + (size_t)myrow));
                t0 = x.x; t1 = x.y; t2 = x.z; t3 = x.w;
            } else {
                const float c = __uint_as_float(in.imm);
                t0 = c; t1 = c; t2 = c; t3 = c;
            }
            continue;
        }
        if (kind == K_UNARY) {
            t0 = rc_unary_f(in.op, t0);
            t1 = rc_unary_f(in.op, t1);
            t2 = rc_unary_f(in.op, t2);
            t3 = rc_unary_f(in.op, t3);
            continue;
        }
        if (kind <= K_BIN_C) {
            float4 av, bv;
            if (kind == K_BIN_S) {
                av = stk[in.arg * T + tid];
                bv = make_float4(t0, t1, t2, t3);
            } else if (kind == K_BIN_V) {
                av = make_float4(t0, t1, t2, t3);
                bv = __ldg(reinterpret_cast<const float4 *>(
                    cols + (size_t)in.imm * (size_t)npad + (size_t)myrow));
            } else {
                const float c = __uint_as_float(in.imm);
                av = make_float4(t0, t1, t2, t3);
                bv = make_float4(c, c, c, c);
            }
            t0 = rc_binary_f(in.op, av.x, bv.x);
            t1 = rc_binary_f(in.op, av.y, bv.y);
            t2 = rc_binary_f(in.op, av.z, bv.z);
            t3 = rc_binary_f(in.op, av.w, bv.w);
            continue;
        }
        if (kind == K_IF) {
            const float4 cnd = stk[in.arg * T + tid];
            const float4 a = stk[(in.arg + 1) * T + tid];
            t0 = cnd.x > 0.0f ? a.x : t0;
            t1 = cnd.y > 0.0f ? a.y : t1;
            t2 = cnd.z > 0.0f ? a.z : t2;
            t3 = cnd.w > 0.0f ? a.w : t3;
            continue;
        }
        if (kind == K_HALT) {
            p = in.arg == 1 ? make_float4(t0, t1, t2, t3) : stk[tid];
            return;
        }
        break;
    }
    p = make_float4(rc_nanf(), rc_nanf(), rc_nanf(), rc_nanf());
}

template <int T>
__global__ void __launch_bounds__(T) rc_score_kernel_wide(ScoreArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    float4 *stk = reinterpret_cast<float4 *>(smem_raw);
    double *sacc = reinterpret_cast<double *>(stk + a.nslots * T);
    double *sacc2 = sacc + a.group * T;
    RcIns *sprog = reinterpret_cast<RcIns *>(sacc2 + a.group * T);
    __shared__ int s_item;
    __shared__ int s_bad;
    const int SUB = T * 4;
    const int mode = a.mode;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= a.nitems) break;
        const int g = item / a.ntiles;
        const int tile = item - g * a.ntiles;
        const int cbase = g * a.group;
        const int gcount = min(a.group, a.ncand - cbase);
        for (int c = 0; c < gcount; ++c) {
            const int cand = a.order[cbase + c];
            const int b = a.ins_off[cand], e = a.ins_off[cand + 1];
            for (int q = tid; q < e - b; q += T) sprog[c * a.maxins + q] = a.ins[b + q];
            sacc[c * T + tid] = 0.0;
            sacc2[c * T + tid] = 0.0;
        }
        if (tid == 0) s_bad = 0;
        unsigned badmask = 0;
        __syncthreads();
        for (int s = 0; s < a.subtiles; ++s) {
            const int row0 = (tile * a.subtiles + s) * SUB;
            if (row0 >= a.n) break;
            const int myrow = row0 + 4 * tid;
            const float4 yv4 = __ldg(reinterpret_cast<const float4 *>(a.y + myrow));
            for (int c = 0; c < gcount; ++c) {
                const int cand = a.order[cbase + c];
                float4 p;
                rc_run_global<T>(sprog + c * a.maxins, a.cols, a.npad, myrow, stk, tid, p);
                double acc = sacc[c * T + tid];
                double acc2 = sacc2[c * T + tid];
                int bad = 0;
                const float pr[4] = {p.x, p.y, p.z, p.w};
                const float yy[4] = {yv4.x, yv4.y, yv4.z, yv4.w};
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int row = myrow + i;
                    if (row < a.n) rc_accumulate<T>(a, mode, pr[i], yy[i], row, cand, acc, acc2, bad);
                }
                sacc[c * T + tid] = acc;
                sacc2[c * T + tid] = acc2;
                if (bad) badmask |= 1u << c;
            }
        }
        __syncthreads();
        if (badmask) atomicOr(&s_bad, (int)badmask);
        for (int st = T / 2; st > 0; st >>= 1) {
            if (tid < st) {
                for (int c = 0; c < gcount; ++c) {
                    if (mode == SM_MAXIMUM) {
                        sacc[c * T + tid] = fmax(sacc[c * T + tid], sacc[c * T + tid + st]);
                    } else {
                        sacc[c * T + tid] += sacc[c * T + tid + st];
                        sacc2[c * T + tid] += sacc2[c * T + tid + st];
                    }
                }
            }
            __syncthreads();
        }
        if (tid < gcount) {
            const int cand = a.order[cbase + tid];
            a.partial[(size_t)cand * a.ptiles + tile] = sacc[tid * T];
            if (a.partial2) a.partial2[(size_t)cand * a.ptiles + tile] = sacc2[tid * T];
            if (s_bad & (1 << tid)) atomicOr(&a.bad[cand], 1);
        }
        __syncthreads();
    }
}

/* Tiles of each candidate in ascending order: the final, fixed-order sum. */
__global__ void rc_score_finalize(int nprog, const int *__restrict__ cand_tiles,
                                  const double *__restrict__ partial,
                                  const double *__restrict__ partial2, int ptiles,
                                  const int *__restrict__ bad, int n, int mode, double syy,
                                  double *__restrict__ out, int *__restrict__ status,
                                  float *__restrict__ out_f32, double *__restrict__ pbar)
{
    const int cand = blockIdx.x * blockDim.x + threadIdx.x;
    if (cand >= nprog) return;
    const int nt = cand_tiles[cand];
    double s = 0.0, s2 = 0.0;
    for (int t = 0; t < nt; ++t) {
        const double v = partial[(size_t)cand * ptiles + t];
        if (mode == SM_MAXIMUM) s = fmax(s, v);
        else s += v;
        if (partial2) s2 += partial2[(size_t)cand * ptiles + t];
    }
    if (mode >= SM_EVAL_SQUARED && mode <= SM_EVAL_ABSOLUTE) {
        out_f32[cand] = (float)s;
        return;
    }
    if (mode == SM_PREDICT) return;
    if (bad[cand]) {
        if (out) out[cand] = INFINITY;
        if (status) status[cand] = RC_SCORE_NONFINITE;
        return;
    }
    const double dn = (double)n;
    double v = 0.0;
    int st = 0;
    switch (mode) {
        case SM_CORR_PASS1:
            pbar[cand] = s / dn;
            return;
        case SM_CORRELATION:
        case SM_CORRELATION_SIGNED: {
            /* s = sum dp^2, s2 = sum dp dy (pass 2); the CPU rule: zero
               variance on either side is rho = 0 (eval.cu:1003-1012). */
            const double rho = (s <= 0.0 || syy <= 0.0) ? 0.0 : s2 / (sqrt(s) * sqrt(syy));
            v = mode == SM_CORRELATION_SIGNED ? 1.0 - rho : 1.0 - fabs(rho);
        } break;
        case SM_AIC: case SM_AICC: case SM_BIC: v = s; break; /* RSS; host penalty */
        case SM_SIGNED: v = fabs(s) / dn; break;
        case SM_MAXIMUM: v = s; break;
        case SM_LOG_LOSS: case SM_BRIER: case SM_HINGE_SIGMOID: case SM_HINGE_ORDINARY:
        case SM_HINGE_SQUARED:
            if (!(s2 > 0.0)) {
                v = INFINITY;
                st = RC_SCORE_ALL_ZERO_WEIGHT;
            } else {
                v = s / s2;
            }
            break;
        default: v = s / dn; break;
    }
    out[cand] = v;
    status[cand] = st;
}

/* ---- host launcher -------------------------------------------------- */

namespace {

struct Bucket {
    std::vector<int> cands;
    int nslots = 0;
    int maxins = 1;
};

int occupancy_blocks(const void *fn, int threads, size_t smem)
{
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return blocks < 1 ? 1 : blocks;
}

/* Rows per tile: fixed per (bucket) so a candidate's reduction order depends
   only on n and its own depth. */
const int TILE_ROWS = 32768;

}  // namespace

static int stage_limit_cols() { return 15; }

float rc_score_run(RcCtx *c, const uint32_t *words, const uint32_t *off, int width, int nprog,
                   int mode, const int *pcount, double *out, int *status, float *out_f32,
                   float *pred_out)
{
    (void)pcount;
    if (!c || nprog <= 0) return -1.0f;
    RcStats *st = &c->stats;
    const double t_begin = rc_now_ms();

    /* 1. decode */
    std::vector<RcIns> ins;
    ins.reserve((size_t)nprog * 16);
    std::vector<int> ins_off(nprog + 1, 0);
    std::vector<int> nslots(nprog, 0);
    std::vector<RcIns> tmp(RC_MAX_INS + 64);
    for (int p = 0; p < nprog; ++p) {
        size_t b = width > 0 ? (size_t)p * (size_t)width : off[p];
        size_t e = width > 0 ? b + (size_t)width : off[p + 1];
        if (e < b) e = b;
        std::vector<RcIns> local(std::max<size_t>(e - b, 1) + 1);
        int ns = 0;
        int cnt = rc_decode_postfix(words + b, e - b, c->v, local.data(), &ns);
        ins_off[p] = (int)ins.size();
        ins.insert(ins.end(), local.begin(), local.begin() + cnt);
        nslots[p] = ns;
    }
    ins_off[nprog] = (int)ins.size();

    /* 2. bucket by depth; longest program first */
    Bucket bk[2];
    for (int p = 0; p < nprog; ++p) {
        const int b = nslots[p] <= RC_SHALLOW_SLOTS ? 0 : 1;
        bk[b].cands.push_back(p);
        bk[b].nslots = std::max(bk[b].nslots, nslots[p]);
        bk[b].maxins = std::max(bk[b].maxins, ins_off[p + 1] - ins_off[p]);
    }
    for (int b = 0; b < 2; ++b) {
        std::stable_sort(bk[b].cands.begin(), bk[b].cands.end(), [&](int x, int y) {
            return (ins_off[x + 1] - ins_off[x]) > (ins_off[y + 1] - ins_off[y]);
        });
    }
    const int Tb[2] = {256, 64};
    const bool staged = (c->v + 1) <= stage_limit_cols() + 1;
    int tiles_b[2], subt_b[2];
    for (int b = 0; b < 2; ++b) {
        const int sub = Tb[b] * 4;
        subt_b[b] = TILE_ROWS / sub;
        tiles_b[b] = (c->n + TILE_ROWS - 1) / TILE_ROWS;
        if (tiles_b[b] < 1) tiles_b[b] = 1;
    }
    const int ptiles = std::max(tiles_b[0], tiles_b[1]);
    std::vector<int> cand_tiles(nprog);
    std::vector<int> order;
    order.reserve(nprog);
    for (int b = 0; b < 2; ++b)
        for (int p : bk[b].cands) {
            cand_tiles[p] = tiles_b[b];
            order.push_back(p);
        }

    const bool corr = (mode == SM_CORRELATION || mode == SM_CORRELATION_SIGNED);
    const bool two = corr || (mode >= SM_LOG_LOSS && mode <= SM_HINGE_SQUARED);

    /* 3. layout: inputs [ins | ins_off | order | cand_tiles] outputs
       [out | status | out_f32] work [partial | partial2 | bad | counters | pbar] */
    size_t cur = 0;
    const size_t o_ins = rc_take(&cur, sizeof(RcIns) * ins.size());
    const size_t o_insoff = rc_take(&cur, sizeof(int) * (nprog + 1));
    const size_t o_order = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_ctiles = rc_take(&cur, sizeof(int) * nprog);
    const size_t in_end = rc_take(&cur, 0);
    const size_t o_out = rc_take(&cur, sizeof(double) * nprog);
    const size_t o_status = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_f32 = rc_take(&cur, sizeof(float) * nprog);
    const size_t io_end = rc_take(&cur, 0);
    const size_t o_part = rc_take(&cur, sizeof(double) * (size_t)nprog * ptiles);
    const size_t o_part2 = rc_take(&cur, two ? sizeof(double) * (size_t)nprog * ptiles : 0);
    const size_t o_bad = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_cnt = rc_take(&cur, sizeof(int) * 8);
    const size_t o_pbar = rc_take(&cur, corr ? sizeof(double) * nprog : 0);
    const size_t o_pred = rc_take(&cur, pred_out ? sizeof(float) * (size_t)nprog * c->n : 0);
    const size_t dev_end = rc_take(&cur, 0);
    double t = rc_now_ms();
    if (rc_reserve(c, dev_end, io_end) != 0) {
        st->failed = 1;
        return -1.0f;
    }
    st->alloc_ms += rc_now_ms() - t;
    unsigned char *dev = c->dev, *host = c->host;
    t = rc_now_ms();
    memcpy(host + o_ins, ins.data(), sizeof(RcIns) * ins.size());
    memcpy(host + o_insoff, ins_off.data(), sizeof(int) * (nprog + 1));
    memcpy(host + o_order, order.data(), sizeof(int) * nprog);
    memcpy(host + o_ctiles, cand_tiles.data(), sizeof(int) * nprog);
    cudaMemcpyAsync(dev, host, in_end, cudaMemcpyHostToDevice, c->s);
    cudaMemsetAsync(dev + o_bad, 0, o_cnt - o_bad + sizeof(int) * 8, c->s);
    st->h2d_ms += rc_now_ms() - t;
    st->h2d_bytes += in_end;

    ScoreArgs a;
    memset(&a, 0, sizeof(a));
    a.cols = c->d_cols;
    a.y = c->d_y;
    a.tsign = c->d_tsign;
    a.w = c->d_w64;
    a.n = c->n;
    a.npad = c->npad;
    a.v = c->v;
    a.ins = reinterpret_cast<const RcIns *>(dev + o_ins);
    a.ins_off = reinterpret_cast<const int *>(dev + o_insoff);
    a.ptiles = ptiles;
    a.partial = reinterpret_cast<double *>(dev + o_part);
    a.partial2 = two ? reinterpret_cast<double *>(dev + o_part2) : nullptr;
    a.bad = reinterpret_cast<int *>(dev + o_bad);
    a.pred = pred_out ? reinterpret_cast<float *>(dev + o_pred) : nullptr;
    a.pbar = corr ? reinterpret_cast<const double *>(dev + o_pbar) : nullptr;
    a.ybar = c->ybar;
    const int *d_ctiles = reinterpret_cast<const int *>(dev + o_ctiles);
    int *d_cnt = reinterpret_cast<int *>(dev + o_cnt);

    t = rc_now_ms();
    cudaEventRecord(c->t0, c->s);
    const int passes = corr ? 2 : 1;
    for (int pass = 0; pass < passes; ++pass) {
        const int kmode = corr ? (pass == 0 ? SM_CORR_PASS1 : SM_CORR_PASS2) : mode;
        if (pass == 1) cudaMemsetAsync(dev + o_bad, 0, sizeof(int) * nprog, c->s);
        int obase = 0;
        for (int b = 0; b < 2; ++b) {
            const int nb = (int)bk[b].cands.size();
            if (nb == 0) continue;
            const int T = Tb[b];
            int group = 8;
            auto it = c->tune.find(b);
            if (it != c->tune.end()) group = it->second.first;
            if (group > nb) group = nb;
            if (group < 1) group = 1;
            a.order = reinterpret_cast<const int *>(dev + o_order) + obase;
            a.ncand = nb;
            a.group = group;
            a.subtiles = subt_b[b];
            a.ntiles = tiles_b[b];
            const int ngroups = (nb + group - 1) / group;
            a.nitems = ngroups * a.ntiles;
            a.maxins = bk[b].maxins;
            a.nslots = std::max(bk[b].nslots, 1);
            a.counter = d_cnt + b + 2 * pass;
            a.mode = kmode;
            size_t smem = (staged ? (size_t)(c->v + 1) * T * 16 : 0) + (size_t)a.nslots * T * 16 +
                          (size_t)group * T * 16 + (size_t)group * a.maxins * sizeof(RcIns);
            const void *fn;
            if (staged) fn = T == 256 ? (const void *)rc_score_kernel<256, true>
                                      : (const void *)rc_score_kernel<64, true>;
            else fn = T == 256 ? (const void *)rc_score_kernel_wide<256>
                               : (const void *)rc_score_kernel_wide<64>;
            if (smem > 48 * 1024) {
                if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem) != cudaSuccess) {
                    cudaGetLastError();
                    st->failed = 1;
                    return -1.0f;
                }
            }
            const int per_sm = occupancy_blocks(fn, T, smem);
            int grid = c->sm_count * per_sm;
            if (grid > a.nitems) grid = a.nitems;
            if (staged) {
                if (T == 256) rc_score_kernel<256, true><<<grid, 256, smem, c->s>>>(a);
                else rc_score_kernel<64, true><<<grid, 64, smem, c->s>>>(a);
            } else {
                if (T == 256) rc_score_kernel_wide<256><<<grid, 256, smem, c->s>>>(a);
                else rc_score_kernel_wide<64><<<grid, 64, smem, c->s>>>(a);
            }
            obase += nb;
        }
        rc_score_finalize<<<(nprog + 127) / 128, 128, 0, c->s>>>(
            nprog, d_ctiles, a.partial, a.partial2, ptiles, a.bad, c->n,
            corr && pass == 1 ? mode : kmode, c->syy,
            reinterpret_cast<double *>(dev + o_out), reinterpret_cast<int *>(dev + o_status),
            reinterpret_cast<float *>(dev + o_f32), reinterpret_cast<double *>(dev + o_pbar));
    }
    cudaEventRecord(c->t1, c->s);
    st->launch_ms += rc_now_ms() - t;
    if (cudaGetLastError() != cudaSuccess) {
        cudaStreamSynchronize(c->s);
        st->failed = 1;
        return -1.0f;
    }
    t = rc_now_ms();
    cudaMemcpyAsync(host + in_end, dev + in_end, io_end - in_end, cudaMemcpyDeviceToHost, c->s);
    if (pred_out) {
        cudaMemcpyAsync(pred_out, dev + o_pred, sizeof(float) * (size_t)nprog * c->n,
                        cudaMemcpyDeviceToHost, c->s);
    }
    if (rc_finish(c) != 0) {
        st->failed = 1;
        return -1.0f;
    }
    st->sync_ms += rc_now_ms() - t;
    t = rc_now_ms();
    if (out) memcpy(out, host + o_out, sizeof(double) * nprog);
    if (status) memcpy(status, host + o_status, sizeof(int) * nprog);
    if (out_f32) memcpy(out_f32, host + o_f32, sizeof(float) * nprog);
    st->d2h_ms += rc_now_ms() - t;
    st->d2h_bytes += io_end - in_end;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->t0, c->t1);
    st->kernel_ms = ms;
    st->batch = nprog;
    st->wall_ms = rc_now_ms() - (c->batch_start_ms > 0 ? c->batch_start_ms : t_begin);
    c->warm = 1;
    c->batches++;
    return ms;
}

/* ---- reference entry points ------------------------------------------ */

static double rc_aic_value(int kind, double rss, int n, int k)
{
    /* metrics.rs:1128-1154 / eval.cu:3626-3640. */
    const double dn = (double)n, dk = (double)k;
    const double base = rss <= 0.0 ? -INFINITY : dn * log(rss / dn);
    if (kind == SM_AIC) return base + 2.0 * dk;
    if (kind == SM_BIC) return base + dk * log(dn);
    if (!std::isfinite(base)) return base;
    const double denom = dn - dk - 1.0;
    if (denom <= 0.0) return INFINITY;
    return base + 2.0 * dk + 2.0 * dk * (dk + 1.0) / denom;
}

static float score_entry(RcCtx *c, const uint32_t *words, const uint32_t *off, int width,
                         int nprog, int kind, const int *pcount, double *out, int *status)
{
    if (kind < 0 || kind > SM_HINGE_SQUARED) return -1.0f;
    if (kind >= SM_LOG_LOSS && !c->has_tsign) return -1.0f;
    float ms = rc_score_run(c, words, off, width, nprog, kind, pcount, out, status, nullptr,
                            nullptr);
    if (ms >= 0.0f && (kind == SM_AIC || kind == SM_AICC || kind == SM_BIC)) {
        for (int i = 0; i < nprog; ++i)
            if (status[i] == 0) out[i] = rc_aic_value(kind, out[i], c->n, pcount ? pcount[i] : 0);
    }
    return ms;
}

extern "C" {

int rc_set_programs(void *ctx, const unsigned int *prog, const unsigned int *off, int nprog)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !prog || !off || nprog <= 0) return -1;
    if (c->pending.active) return -1;
    const size_t words = off[nprog];
    c->prog_words.assign(prog, prog + words);
    c->prog_off.assign(off, off + nprog + 1);
    c->nprog = nprog;
    c->stats.batch = nprog;
    return 0;
}

int rc_eval_submit(void *ctx, int loss)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || c->nprog <= 0 || c->pending.active) return -1;
    if (loss != 0 && loss != 1 && loss != 4) return -1;
    c->pending.active = 1;
    c->pending.nprog = c->nprog;
    c->pending.loss = loss;
    return 0;
}

float rc_eval_collect(void *ctx, float *out)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !out || !c->pending.active) return -1.0f;
    c->pending.active = 0;
    return rc_score_run(c, c->prog_words.data(), c->prog_off.data(), 0, c->pending.nprog,
                        SM_EVAL_SQUARED + c->pending.loss, nullptr, nullptr, nullptr, out,
                        nullptr);
}

float rc_eval(void *ctx, float *out, int loss)
{
    if (rc_eval_submit(ctx, loss) != 0) return -1.0f;
    return rc_eval_collect(ctx, out);
}

float rc_score_batch(void *ctx, const unsigned int *prog, const unsigned int *off, int nprog,
                     int kind, const int *pcount, double *out, int *status)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !prog || !off || nprog <= 0 || !out || !status) return -1.0f;
    if (rc_set_programs(ctx, prog, off, nprog) != 0) return -1.0f;
    return score_entry(c, prog, off, 0, nprog, kind, pcount, out, status);
}

int rc_predict(void *ctx, const unsigned int *prog, const unsigned int *off, int nprog,
               float *out)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !prog || !off || nprog <= 0 || !out) return -1;
    if (rc_set_programs(ctx, prog, off, nprog) != 0) return -1;
    float ms = rc_score_run(c, prog, off, 0, nprog, SM_PREDICT, nullptr, nullptr, nullptr,
                            nullptr, out);
    return ms >= 0.0f ? 0 : -1;
}

int rc_pool_reserve(void *ctx, int nprog, int width)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || nprog <= 0 || width <= 0) return -1;
    if (c->pool_cap >= nprog && c->pool_width == width) return 0;
    for (int i = 0; i < 2; ++i) {
        if (c->d_pool[i]) cudaFree(c->d_pool[i]);
        c->d_pool[i] = nullptr;
        c->alloc_calls++;
        if (c->warm) c->steady_alloc_calls++;
    }
    const size_t bytes = sizeof(unsigned int) * (size_t)nprog * (size_t)width;
    for (int i = 0; i < 2; ++i) {
        if (cudaMalloc((void **)&c->d_pool[i], bytes) != cudaSuccess) {
            cudaGetLastError();
            c->stats.failed = 1;
            return -1;
        }
        c->alloc_calls++;
        if (c->warm) c->steady_alloc_calls++;
        c->pool_host[i].assign((size_t)nprog * width, (uint32_t)OP_HALT);
    }
    c->pool_cap = nprog;
    c->pool_width = width;
    return 0;
}

int rc_pool_upload(void *ctx, int which, const unsigned int *prog, int nprog)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !prog || nprog <= 0 || nprog > c->pool_cap) return -1;
    const int b = which & 1;
    if (!c->d_pool[b]) return -1;
    const size_t words = (size_t)nprog * (size_t)c->pool_width;
    memcpy(c->pool_host[b].data(), prog, sizeof(uint32_t) * words);
    const double t = rc_now_ms();
    if (cudaMemcpy(c->d_pool[b], prog, sizeof(uint32_t) * words, cudaMemcpyHostToDevice) !=
        cudaSuccess)
        return -1;
    c->stats.h2d_ms += rc_now_ms() - t;
    c->stats.h2d_bytes += sizeof(uint32_t) * words;
    c->stats.batch = nprog;
    return 0;
}

float rc_pool_eval(void *ctx, int which, int nprog, int width, float *out, int loss)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !out || nprog <= 0 || nprog > c->pool_cap || width != c->pool_width) return -1.0f;
    if (loss != 0 && loss != 1 && loss != 4) return -1.0f;
    return rc_score_run(c, c->pool_host[which & 1].data(), nullptr, width, nprog,
                        SM_EVAL_SQUARED + loss, nullptr, nullptr, nullptr, out, nullptr);
}

float rc_pool_score(void *ctx, int which, int nprog, int width, int kind, const int *pcount,
                    double *out, int *status)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !out || !status || nprog <= 0 || nprog > c->pool_cap || width != c->pool_width)
        return -1.0f;
    return score_entry(c, c->pool_host[which & 1].data(), nullptr, width, nprog, kind, pcount,
                       out, status);
}

}  // extern "C"

/* FNV-1a of each pool slot up to and including HALT (eval.cu:2665-2681,
   genome.rs:43). */
__global__ void rc_hash_kernel(const unsigned int *__restrict__ prog, int width, int nprog,
                               unsigned long long *__restrict__ out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nprog) return;
    const unsigned int *slot = prog + (size_t)p * (size_t)width;
    unsigned long long h = 0xcbf29ce484222325ULL;
    for (int q = 0; q < width; ++q) {
        const unsigned int w = slot[q];
        h ^= (unsigned long long)w;
        h *= 0x00000100000001b3ULL;
        if (w == OP_HALT) break;
    }
    out[p] = h;
}

extern "C" int rc_pool_hash(void *ctx, int which, int nprog, int width, unsigned long long *out)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !out || nprog <= 0 || nprog > c->pool_cap || width != c->pool_width) return -1;
    const int b = which & 1;
    if (!c->d_pool[b]) return -1;
    size_t cur = 0;
    const size_t o = rc_take(&cur, sizeof(unsigned long long) * nprog);
    if (rc_reserve(c, cur, cur) != 0) return -1;
    rc_hash_kernel<<<(nprog + 127) / 128, 128, 0, c->s>>>(
        c->d_pool[b], width, nprog, reinterpret_cast<unsigned long long *>(c->dev + o));
    cudaMemcpyAsync(c->host + o, c->dev + o, sizeof(unsigned long long) * nprog,
                    cudaMemcpyDeviceToHost, c->s);
    if (rc_finish(c) != 0) return -1;
    memcpy(out, c->host + o, sizeof(unsigned long long) * nprog);
    return 0;
}

/* ======================================================================
 * Scoring without any allocation.
 *
 * Some callers cannot call cudaMalloc at all: a host application whose
 * device memory belongs to another allocator (a caching pool that must not
 * be bypassed or fragmented), or a pipelined search loop on its own streams
 * where cudaMalloc/cudaFree would synchronise the whole device and stall
 * the work in flight. rc_score_batch_noalloc serves them: the caller owns
 * every input and output buffer on the device, and the kernel's scratch
 * (decoded programs, per-tile partial sums, flags, the work counter) lives
 * in one file-scope __device__ array of RC_NOALLOC_SCRATCH_BYTES, which
 * every GPU that loads this library holds until the process exits.
 *
 * All calls share that array and it keeps the previous call's contents:
 * the counter and flags are cleared at the start of every call, and two
 * calls that overlap on the GPU (different streams, or host threads racing
 * on one device) race on the scratch and produce garbage. Serialise them.
 * ====================================================================== */

#define RC_NOALLOC_SCRATCH_BYTES (16u << 20)
#define RC_NOALLOC_MAX_DEVICES 64
#define RC_NOALLOC_TOO_DEEP 3

static __device__ __align__(256) unsigned char rc_noalloc_scratch[RC_NOALLOC_SCRATCH_BYTES];

/* Device-side decoder: one thread per program, the same translation as the
   host decoder (rc_decode_postfix) into a fixed stride of RC_MAX_INS
   instructions. A program needing more than RC_SHALLOW_SLOTS spill slots is
   replaced by K_NAN and flagged `deep`. */
__global__ void rc_noalloc_decode(const unsigned int *__restrict__ prog,
                                  const unsigned int *__restrict__ off, int nprog, int v,
                                  RcIns *__restrict__ ins, int *__restrict__ ins_off,
                                  int *__restrict__ order, int *__restrict__ cand_tiles,
                                  int *__restrict__ deep, int ntiles)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > nprog) return;
    ins_off[p] = p * RC_MAX_INS;
    if (p == nprog) return;
    order[p] = p;
    cand_tiles[p] = ntiles;
    deep[p] = 0;
    RcIns *out = ins + (size_t)p * RC_MAX_INS;
    const unsigned int b = off[p], e = off[p + 1];
    int depth = 0, maxslot = -1, n = 0;
    bool ok = e >= b, halted = false;
    unsigned int i = b;
    while (ok && i < e) {
        const unsigned int w = prog[i++];
        RcIns in;
        in.kind = 0;
        in.op = 0;
        in.arg = 0;
        in.spill = 0xff;
        in.imm = 0;
        if (w == OP_CONST || w == OP_VAR) {
            if (i >= e || depth >= RC_MAX_STACK) { ok = false; break; }
            const unsigned int a = prog[i++];
            if (w == OP_VAR && (long long)a >= (long long)v) { ok = false; break; }
            in.kind = w == OP_CONST ? K_PUSH_CONST : K_PUSH_VAR;
            in.spill = depth >= 1 ? (uint8_t)(depth - 1) : 0xff;
            in.imm = a;
            if (depth >= 1 && depth - 1 > maxslot) maxslot = depth - 1;
            ++depth;
        } else if (w == OP_HALT) {
            if (depth < 1) { ok = false; break; }
            in.kind = K_HALT;
            in.arg = depth == 1 ? 1 : 0;
            halted = true;
        } else if (w == OP_ADD || w == OP_SUB || w == OP_MUL || w == OP_DIV || w == OP_POW ||
                   w == OP_MOD || w == OP_ATAN2 || w == OP_MIN || w == OP_MAX ||
                   w == OP_EQUAL || w == OP_LESS || w == OP_LESS_OR_EQUAL ||
                   w == OP_GREATER || w == OP_GREATER_OR_EQUAL || w == OP_AND || w == OP_OR ||
                   w == OP_XOR) {
            if (depth < 2) { ok = false; break; }
            in.kind = K_BIN_S;
            in.op = (uint8_t)w;
            in.arg = (uint8_t)(depth - 2);
            --depth;
            const bool fus = w == OP_ADD || w == OP_SUB || w == OP_MUL || w == OP_DIV ||
                             w == OP_POW;
            if (n > 0 && fus) {
                RcIns &prev = out[n - 1];
                if ((prev.kind == K_PUSH_VAR || prev.kind == K_PUSH_CONST) &&
                    prev.spill != 0xff && prev.spill == in.arg) {
                    prev.kind = prev.kind == K_PUSH_VAR ? K_BIN_V : K_BIN_C;
                    prev.op = (uint8_t)w;
                    prev.spill = 0xff;
                    continue;
                }
            }
        } else if (w == OP_IF) {
            if (depth < 3) { ok = false; break; }
            in.kind = K_IF;
            in.arg = (uint8_t)(depth - 3);
            depth -= 2;
        } else {
            if (depth < 1) { ok = false; break; }
            in.kind = K_UNARY;
            in.op = w > 253 ? 254 : (uint8_t)w;
        }
        if (n >= RC_MAX_INS) { ok = false; break; }
        out[n++] = in;
        if (halted) break;
    }
    if (!ok || !halted || maxslot + 1 > RC_SHALLOW_SLOTS) {
        deep[p] = ok && halted ? 1 : 0;
        RcIns bad;
        bad.kind = K_NAN;
        bad.op = 0;
        bad.arg = 0;
        bad.spill = 0xff;
        bad.imm = 0;
        out[0] = bad;
    }
}

__global__ void rc_noalloc_mark_deep(int nprog, const int *__restrict__ deep,
                                     double *__restrict__ out, int *__restrict__ status)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < nprog && deep[p]) {
        out[p] = CUDART_NAN;
        status[p] = RC_NOALLOC_TOO_DEEP;
    }
}

namespace {
struct NoallocDevice {
    int ready;
    unsigned char *scratch; /* device address of rc_noalloc_scratch */
    int sm_count;
    int grid_per_sm;
};
NoallocDevice g_noalloc[RC_NOALLOC_MAX_DEVICES];
std::mutex g_noalloc_mu;
}  // namespace

extern "C" int rc_score_batch_noalloc(const float *cols, const float *y, int n, int v, int ld,
                                      const unsigned int *prog, const unsigned int *off,
                                      int nprog, int kind, double *out, int *status,
                                      void *stream)
{
    const int T = 256;
    const int SUB = T * 4;
    if (!cols || !y || !prog || !off || !out || !status || n <= 0 || v <= 0 || nprog <= 0) {
        fprintf(stderr, "rc_score_batch_noalloc: null pointer or empty size\n");
        return -3;
    }
    if (kind < SM_SQUARED || kind > SM_MAXIMUM) {
        fprintf(stderr, "rc_score_batch_noalloc: kind %d unsupported (0..4 only)\n", kind);
        return -3;
    }
    if (v + 1 > stage_limit_cols() + 1) {
        fprintf(stderr, "rc_score_batch_noalloc: %d columns exceed the staged limit %d\n", v,
                stage_limit_cols());
        return -3;
    }
    const long long need_rows = ((long long)n + SUB - 1) / SUB * SUB;
    if ((long long)ld < need_rows || (ld % 4) != 0 || ((uintptr_t)cols % 16) != 0 ||
        ((uintptr_t)y % 16) != 0) {
        fprintf(stderr,
                "rc_score_batch_noalloc: ld must be a multiple of 4 and >= %lld (n rounded up "
                "to %d rows, readable), cols and y 16-byte aligned\n",
                need_rows, SUB);
        return -3;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= RC_NOALLOC_MAX_DEVICES) {
        cudaGetLastError();
        return -1;
    }
    const int ntiles = (int)((n + TILE_ROWS - 1) / TILE_ROWS);
    size_t cur = 0;
    const size_t o_ins = rc_take(&cur, sizeof(RcIns) * (size_t)nprog * RC_MAX_INS);
    const size_t o_insoff = rc_take(&cur, sizeof(int) * ((size_t)nprog + 1));
    const size_t o_order = rc_take(&cur, sizeof(int) * (size_t)nprog);
    const size_t o_ctiles = rc_take(&cur, sizeof(int) * (size_t)nprog);
    const size_t o_deep = rc_take(&cur, sizeof(int) * (size_t)nprog);
    const size_t o_part = rc_take(&cur, sizeof(double) * (size_t)nprog * ntiles);
    const size_t o_bad = rc_take(&cur, sizeof(int) * (size_t)nprog);
    const size_t o_cnt = rc_take(&cur, sizeof(int) * 8);
    const size_t need = rc_take(&cur, 0);
    if (need > RC_NOALLOC_SCRATCH_BYTES) {
        fprintf(stderr,
                "rc_score_batch_noalloc: %d programs over %d rows need %zu scratch bytes, the "
                "static maximum is %u\n",
                nprog, n, need, RC_NOALLOC_SCRATCH_BYTES);
        return -2;
    }
    const int G = 8;
    const size_t smem = (size_t)(v + 1) * T * 16 + (size_t)RC_SHALLOW_SLOTS * T * 16 +
                        (size_t)G * T * 16 + (size_t)G * RC_MAX_INS * sizeof(RcIns);
    NoallocDevice *d = &g_noalloc[dev];
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!d->ready) {
            void *ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, rc_noalloc_scratch);
            if (e != cudaSuccess || !ptr) {
                fprintf(stderr, "rc_score_batch_noalloc: cudaGetSymbolAddress failed: %s\n",
                        cudaGetErrorString(e));
                cudaGetLastError();
                return -1;
            }
            const int maxsmem = (int)((size_t)(stage_limit_cols() + 1) * T * 16 +
                                      (size_t)RC_SHALLOW_SLOTS * T * 16 + (size_t)G * T * 16 +
                                      (size_t)G * RC_MAX_INS * sizeof(RcIns));
            if (cudaFuncSetAttribute((const void *)rc_score_kernel<256, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     maxsmem) != cudaSuccess) {
                cudaGetLastError();
                return -1;
            }
            int sms = 1, per = 1;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &per, rc_score_kernel<256, true>, T, (size_t)maxsmem) != cudaSuccess) {
                cudaGetLastError();
                per = 1;
            }
            d->scratch = (unsigned char *)ptr;
            d->sm_count = sms > 0 ? sms : 1;
            d->grid_per_sm = per > 0 ? per : 1;
            d->ready = 1;
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char *sc = d->scratch;
    cudaMemsetAsync(sc + o_bad, 0, o_cnt - o_bad + sizeof(int) * 8, s);
    rc_noalloc_decode<<<(nprog + 1 + 127) / 128, 128, 0, s>>>(
        prog, off, nprog, v, reinterpret_cast<RcIns *>(sc + o_ins),
        reinterpret_cast<int *>(sc + o_insoff), reinterpret_cast<int *>(sc + o_order),
        reinterpret_cast<int *>(sc + o_ctiles), reinterpret_cast<int *>(sc + o_deep), ntiles);
    ScoreArgs a;
    memset(&a, 0, sizeof(a));
    a.cols = cols;
    a.y = y;
    a.n = n;
    a.npad = ld;
    a.v = v;
    a.ins = reinterpret_cast<const RcIns *>(sc + o_ins);
    a.ins_off = reinterpret_cast<const int *>(sc + o_insoff);
    a.order = reinterpret_cast<const int *>(sc + o_order);
    a.ncand = nprog;
    a.group = G < nprog ? G : nprog;
    a.subtiles = TILE_ROWS / SUB;
    a.ntiles = ntiles;
    a.nitems = ((nprog + a.group - 1) / a.group) * ntiles;
    a.maxins = RC_MAX_INS;
    a.nslots = RC_SHALLOW_SLOTS;
    a.counter = reinterpret_cast<int *>(sc + o_cnt);
    a.partial = reinterpret_cast<double *>(sc + o_part);
    a.partial2 = nullptr;
    a.ptiles = ntiles;
    a.bad = reinterpret_cast<int *>(sc + o_bad);
    a.mode = kind;
    int grid = d->sm_count * d->grid_per_sm;
    if (grid > a.nitems) grid = a.nitems;
    rc_score_kernel<256, true><<<grid, T, smem, s>>>(a);
    rc_score_finalize<<<(nprog + 127) / 128, 128, 0, s>>>(
        nprog, reinterpret_cast<const int *>(sc + o_ctiles), a.partial, nullptr, ntiles, a.bad, n,
        kind, 0.0, out, status, nullptr, nullptr);
    rc_noalloc_mark_deep<<<(nprog + 127) / 128, 128, 0, s>>>(
        nprog, reinterpret_cast<const int *>(sc + o_deep), out, status);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "rc_score_batch_noalloc: launch failed: %s\n", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}
