/*
 * The exact f64 finalist refit and the structure-of-arrays evaluator, on the
 * host cores.
 *
 * After the device fit, every reported finalist is refit exactly in f64 by
 * the caller's CPU code (`refit_finalists_exact`, my-version/src/fit/gpu.rs:
 * 666-687): `fit_lm` for the least-squares family (fit.rs:2534-2624) and the
 * IRLS arms of `fit_weighted_metric` for absolute and log-squashed
 * (fit.rs:2937-2974, :3092-3170). The reference walks one row at a time
 * (`eval_row`, `backward`, fit.rs:1424-1671). Here the same arithmetic runs
 * over blocks of RB rows node by node: a post-order program is evaluated
 * column-wise into a [node][RB] value block, the adjoint sweep runs over the
 * block the same way, and the normal equations, SSE and scores are then
 * accumulated row by row in row order. Every per-row value is produced by the
 * same f64 operation as the row walk and every sum is taken in the same order,
 * so the refit is bit-identical to the reference's; only the loop nest
 * differs (the node switch is taken once per block, and the element-wise
 * arithmetic vectorises). Finalists run concurrently on teams of threads:
 * one thread each when there are at least as many finalists as threads,
 * otherwise a finalist's passes are split by rows over its team (rows
 * block-parallel, then every sum in row order on one thread). The thread
 * count never changes a bit.
 *
 * The evaluator has the reference's two sets of domain rules: the tree
 * evaluator's (`expr::eval`, which `eval_soa.rs:273-380` mirrors: guarded
 * ln / sqrt / tan / pow / atan2), used for predictions and scores, and the
 * flat evaluator's (`value_of`, fit.rs:1211-1382), used inside the LM.
 *
 * Trees arrive as pre-order (op, val) arrays with the device opcodes (0..42,
 * 64..66 for the inverse hyperbolics); inputs are column-major f64
 * `cols[var * n + row]`. Exposed as the C functions in include/rcsr_refit.h.
 *
 * Compile without value-changing floating-point options (no -ffast-math,
 * -ffp-contract=off): the bit-identity rests on IEEE element-wise arithmetic.
 */
#include "rcsr_refit.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include <omp.h>

namespace {

enum {
    CONST = 0, VAR = 1, ADD = 2, SUB = 3, MUL = 4, DIV = 5, SIN = 6, COS = 7, TAN = 8, EXP = 9,
    LOG = 10, SQRT = 11, ABS = 12, TANH = 13, SIG = 14, SQUARE = 15, CUBE = 16, NEG = 17,
    GAUSS = 18, STEP = 19, POW = 20, SINH = 21, COSH = 22, FLOOR = 23, CEIL = 24, ROUND = 25,
    MOD = 26, ATAN2 = 27, ERF = 28, ERFC = 29, MIN = 30, MAX = 31, IF = 32, SIGN = 33,
    EQUAL = 34, LESS = 35, LESS_OR_EQUAL = 36, GREATER = 37, GREATER_OR_EQUAL = 38, AND = 39,
    OR = 40, XOR = 41, NOT = 42, ASINH = 64, ACOSH = 65, ATANH = 66
};

/* metrics.rs metric codes (the same numbering as the device score kinds'
   callers use). */
enum {
    MT_SQUARED = 0, MT_ABSOLUTE = 1, MT_LOG_SQUASHED = 2, MT_AIC = 7, MT_AICC = 8, MT_BIC = 9
};

constexpr int RB = 256; /* rows per block */
const double INF = std::numeric_limits<double>::infinity();
const double NaN = std::numeric_limits<double>::quiet_NaN();
const double INV_SQRT_PI = 0.56418958354775628695;

int arity(int op)
{
    switch (op) {
        case CONST: case VAR: return 0;
        case ADD: case SUB: case MUL: case DIV: case POW: case MOD: case ATAN2: case MIN:
        case MAX: case EQUAL: case LESS: case LESS_OR_EQUAL: case GREATER:
        case GREATER_OR_EQUAL: case AND: case OR: case XOR: return 2;
        case IF: return 3;
        default: return 1;
    }
}

/* A tree as a post-order program (fit.rs:1068-1196 `flatten`): node i's
   operands are earlier nodes; every constant leaf owns the next slot, so the
   slot order is the constants' left-to-right order, which is also the order
   of their pre-order positions (`cpos`). */
struct Prog {
    std::vector<int> op, k0, k1, k2, nk, slot;
    std::vector<double> val;
    std::vector<int> cpos;
    std::vector<char> live; /* a constant lies in the node's subtree */
    int root = 0;
    int size() const { return (int)op.size(); }
};

int lay(const int *ops, const double *vals, int nn, int &pos, int depth, Prog &p)
{
    if (pos >= nn || depth > 4096) return -1;
    const int me = pos++;
    const int o = ops[me];
    int kid[3] = {0, 0, 0};
    const int a = arity(o);
    for (int i = 0; i < a; ++i) {
        kid[i] = lay(ops, vals, nn, pos, depth + 1, p);
        if (kid[i] < 0) return -1;
    }
    p.op.push_back(o);
    p.val.push_back(vals[me]);
    p.k0.push_back(kid[0]);
    p.k1.push_back(kid[1]);
    p.k2.push_back(kid[2]);
    p.nk.push_back(a);
    bool live = o == CONST;
    for (int i = 0; i < a; ++i) live = live || p.live[kid[i]];
    p.live.push_back(live ? 1 : 0);
    if (o == CONST) {
        p.slot.push_back((int)p.cpos.size());
        p.cpos.push_back(me);
    } else {
        p.slot.push_back(-1);
    }
    return p.size() - 1;
}

bool load(const int *ops, const double *vals, int nn, Prog &p)
{
    int pos = 0;
    const int r = lay(ops, vals, nn, pos, 0, p);
    if (r < 0 || pos != nn) return false;
    p.root = r;
    return true;
}

/* ---- the reference's special functions ---------------------------------------- */

/* erf / erfc through the regularised incomplete gamma of order 1/2
   (expr.rs:930-1041): the series below x = 1.5, Lentz's continued fraction
   above, at most 300 terms, tolerance 1e-15. */
const double ERF_TOL = 1e-15;
const double ERF_TINY = 1e-300;

double half_gamma_cf(double x)
{
    const double a = 0.5;
    double b = x + 1.0 - a, c = 1.0 / ERF_TINY, d = 1.0 / b, h = d;
    for (int i = 1; i < 300; ++i) {
        const double an = -(double)i * ((double)i - a);
        b += 2.0;
        d = an * d + b;
        if (std::fabs(d) < ERF_TINY) d = ERF_TINY;
        c = b + an / c;
        if (std::fabs(c) < ERF_TINY) c = ERF_TINY;
        d = 1.0 / d;
        const double del = d * c;
        h *= del;
        if (std::fabs(del - 1.0) < ERF_TOL) break;
    }
    return std::exp(-x + a * std::log(x) - 0.5 * std::log(M_PI)) * h;
}

/* Rust's clamp(0, 1): a NaN stays NaN. */
double unit_clamp(double v)
{
    if (v < 0.0) v = 0.0;
    if (v > 1.0) v = 1.0;
    return v;
}

double half_gamma_p(double x)
{
    if (std::isnan(x)) return NaN;
    if (x <= 0.0) return 0.0;
    if (!std::isfinite(x)) return 1.0;
    if (x >= 1.5) return unit_clamp(1.0 - half_gamma_cf(x));
    const double a = 0.5;
    double ap = a, sum = 1.0 / a, del = sum;
    for (int i = 0; i < 300; ++i) {
        ap += 1.0;
        del *= x / ap;
        sum += del;
        if (std::fabs(del) < std::fabs(sum) * ERF_TOL) break;
    }
    return unit_clamp(sum * std::exp(-x + a * std::log(x) - 0.5 * std::log(M_PI)));
}

double half_gamma_q(double x)
{
    if (std::isnan(x)) return NaN;
    if (x <= 0.0) return 1.0;
    if (!std::isfinite(x)) return 0.0;
    if (x < 1.5) return unit_clamp(1.0 - half_gamma_p(x));
    return unit_clamp(half_gamma_cf(x));
}

double ref_erf(double x)
{
    if (std::isnan(x)) return NaN;
    const double p = half_gamma_p(x * x);
    return x < 0.0 ? -p : p;
}

double ref_erfc(double x)
{
    if (std::isnan(x)) return NaN;
    const double q = half_gamma_q(x * x);
    return x < 0.0 ? 2.0 - q : q;
}

/* Rust std's f64::asinh / acosh / atanh (the published forms the tree
   evaluator calls, expr.rs:1181-1200). */
double ref_asinh(double x)
{
    const double ax = std::fabs(x), inv = 1.0 / ax;
    return std::copysign(std::log1p(ax + ax / (std::hypot(1.0, inv) + inv)), x);
}

double ref_acosh(double x)
{
    if (x < 1.0) return NaN;
    return std::log(x + std::sqrt(x - 1.0) * std::sqrt(x + 1.0));
}

double ref_atanh(double x) { return 0.5 * std::log1p((2.0 * x) / (1.0 - x)); }

double compare(double a, double b, int op)
{
    if (std::isnan(a) || std::isnan(b)) return NaN;
    bool t;
    switch (op) {
        case EQUAL: t = a == b; break;
        case LESS: t = a < b; break;
        case LESS_OR_EQUAL: t = a <= b; break;
        case GREATER: t = a > b; break;
        default: t = a >= b; break;
    }
    return t ? 1.0 : 0.0;
}

double logic(double a, double b, int op)
{
    if (std::isnan(a) || std::isnan(b)) return NaN;
    const bool x = a > 0.0, y = b > 0.0;
    bool t;
    switch (op) {
        case AND: t = x && y; break;
        case OR: t = x || y; break;
        default: t = x != y; break;
    }
    return t ? 1.0 : 0.0;
}

/* ---- per-element rules ------------------------------------------------------ */

/* One unary node. TREE selects `expr::eval`'s guards, otherwise the flat
   evaluator's `value_of`. */
template <bool TREE>
inline double unary(int op, double x)
{
    switch (op) {
        case NEG: return -x;
        case EXP: return x > 700.0 ? INF : std::exp(x);
        case LOG:
            if (TREE) return x > 0.0 ? std::log(x) : NaN;
            return std::log(x);
        case ABS: return std::fabs(x);
        case SQRT:
            if (TREE) return x >= 0.0 ? std::sqrt(x) : NaN;
            return std::sqrt(x);
        case SIN: return std::sin(x);
        case COS: return std::cos(x);
        case TAN: {
            const double t = std::tan(x);
            if (TREE) return std::isfinite(t) ? t : NaN;
            return t;
        }
        case SINH: return std::sinh(x);
        case COSH: return std::cosh(x);
        case TANH: return std::tanh(x);
        case SIG: return 1.0 / (1.0 + std::exp(-x));
        case STEP: return x > 0.0 ? 1.0 : 0.0;
        case GAUSS: return std::exp(-x * x);
        case SQUARE: return x * x;
        case CUBE: return x * x * x;
        case FLOOR: return std::floor(x);
        case CEIL: return std::ceil(x);
        case ROUND: return std::round(x);
        case SIGN:
            if (x > 0.0) return 1.0;
            if (x < 0.0) return -1.0;
            if (x == 0.0) return 0.0;
            return NaN;
        case ERF: return ref_erf(x);
        case ERFC: return ref_erfc(x);
        case ASINH: return ref_asinh(x);
        case ACOSH: return x >= 1.0 ? ref_acosh(x) : NaN;
        case ATANH: return std::fabs(x) < 1.0 ? ref_atanh(x) : NaN;
        case NOT:
            if (std::isnan(x)) return NaN;
            return x > 0.0 ? 0.0 : 1.0;
        default: return NaN;
    }
}

template <bool TREE>
inline double binary(int op, double a, double b)
{
    switch (op) {
        case ADD: return a + b;
        case SUB: return a - b;
        case MUL: return a * b;
        case DIV: return std::fabs(b) < 1e-12 ? NaN : a / b;
        case POW:
            if (TREE && a < 0.0 && std::fabs(b - std::round(b)) > 1e-9) return NaN;
            return std::pow(a, b);
        case MOD:
            if (!std::isfinite(a) || !std::isfinite(b) || std::fabs(b) < 1e-12) return NaN;
            return a - b * std::floor(a / b);
        case MIN:
            if (std::isnan(a) || std::isnan(b)) return NaN;
            return std::fmin(a, b);
        case MAX:
            if (std::isnan(a) || std::isnan(b)) return NaN;
            return std::fmax(a, b);
        case ATAN2:
            if (TREE && (std::isnan(a) || std::isnan(b))) return NaN;
            return std::atan2(a, b);
        case EQUAL: case LESS: case LESS_OR_EQUAL: case GREATER: case GREATER_OR_EQUAL:
            return compare(a, b, op);
        case AND: case OR: case XOR: return logic(a, b, op);
        default: return NaN;
    }
}

inline double indicator(double x)
{
    if (std::isnan(x)) return NaN;
    return x > 0.0 ? 1.0 : 0.0;
}

/* ---- block sweeps ------------------------------------------------------------ */

struct Data {
    const double *cols;
    int64_t n;
    int nv;
    const double *y;
    const double *w; /* null: every row weighs 1 */
};

/* Where a flat sweep takes each node from: evaluated, copied from the
   fit's cache of constant-free subtree values, or not needed (inside a
   cached subtree). */
enum { NODE_EVAL = 0, NODE_CACHED = 1, NODE_SKIP = 2 };

struct Plan {
    std::vector<char> mode;
    std::vector<int> col;      /* cache column of a NODE_CACHED node */
    std::vector<double> cache; /* [column][n] */
};

/* Values of every node over rows [r0, r0 + nb) into V[node][RB]. `c` holds
   the constants by slot (null: the tree's own values). With a plan, cached
   constant-free subtrees are copied instead of evaluated. */
template <bool TREE>
void forward(const Prog &p, const Data &d, int64_t r0, int nb, const double *c, double *V,
             const Plan *plan = nullptr)
{
    const int m = p.size();
    for (int i = 0; i < m; ++i) {
        double *o = V + (size_t)i * RB;
        if (plan && plan->mode[i] != NODE_EVAL) {
            if (plan->mode[i] == NODE_CACHED)
                std::memcpy(o, plan->cache.data() + (size_t)plan->col[i] * (size_t)d.n + r0,
                            sizeof(double) * (size_t)nb);
            continue;
        }
        const double *a = V + (size_t)p.k0[i] * RB;
        const double *b = V + (size_t)p.k1[i] * RB;
        const double *e = V + (size_t)p.k2[i] * RB;
        const int op = p.op[i];
        switch (op) {
            case CONST: {
                const double v = (c && p.slot[i] >= 0) ? c[p.slot[i]] : p.val[i];
                for (int r = 0; r < nb; ++r) o[r] = v;
            } break;
            case VAR: {
                const double fv = p.val[i];
                const long idx = (long)fv;
                if (fv >= 0 && idx < d.nv) {
                    const double *col = d.cols + (size_t)idx * (size_t)d.n + (size_t)r0;
                    std::memcpy(o, col, sizeof(double) * (size_t)nb);
                } else {
                    for (int r = 0; r < nb; ++r) o[r] = NaN;
                }
            } break;
            case ADD: for (int r = 0; r < nb; ++r) o[r] = a[r] + b[r]; break;
            case SUB: for (int r = 0; r < nb; ++r) o[r] = a[r] - b[r]; break;
            case MUL: for (int r = 0; r < nb; ++r) o[r] = a[r] * b[r]; break;
            case DIV:
                for (int r = 0; r < nb; ++r) o[r] = std::fabs(b[r]) < 1e-12 ? NaN : a[r] / b[r];
                break;
            case NEG: for (int r = 0; r < nb; ++r) o[r] = -a[r]; break;
            case ABS: for (int r = 0; r < nb; ++r) o[r] = std::fabs(a[r]); break;
            case SQUARE: for (int r = 0; r < nb; ++r) o[r] = a[r] * a[r]; break;
            case CUBE: for (int r = 0; r < nb; ++r) o[r] = a[r] * a[r] * a[r]; break;
            case IF:
                for (int r = 0; r < nb; ++r) o[r] = a[r] > 0.0 ? b[r] : e[r];
                break;
            default:
                if (p.nk[i] == 2) {
                    for (int r = 0; r < nb; ++r) o[r] = binary<TREE>(op, a[r], b[r]);
                } else if (p.nk[i] == 1) {
                    for (int r = 0; r < nb; ++r) o[r] = unary<TREE>(op, a[r]);
                } else {
                    for (int r = 0; r < nb; ++r) o[r] = NaN;
                }
                break;
        }
    }
}

/* The reverse-mode adjoint over the block (fit.rs:1453-1671 `backward`),
   seeded with 1 at the root; G[slot][RB] receives d f / d c_slot. A node
   whose adjoint is zero passes nothing on, exactly as the row sweep skips
   it. Where a partial is a function the forward block already evaluated at
   the same argument (exp, the logistic, tanh, the Gaussian, sqrt, pow), the
   node's own value is read instead of calling the function again: the same
   function of the same argument, so the same bits. */
void backward(const Prog &p, int nb, const double *V, double *A, double *G)
{
    const int m = p.size();
    std::fill(A, A + (size_t)m * RB, 0.0);
    for (int r = 0; r < nb; ++r) A[(size_t)p.root * RB + r] = 1.0;
    for (int i = m - 1; i >= 0; --i) {
        /* below a node without constants nothing reaches G */
        if (!p.live[i]) continue;
        const double *ad = A + (size_t)i * RB;
        const int op = p.op[i];
        if (op == CONST) {
            if (p.slot[i] >= 0) {
                double *g = G + (size_t)p.slot[i] * RB;
                for (int r = 0; r < nb; ++r) g[r] = ad[r] == 0.0 ? 0.0 : 0.0 + ad[r];
            }
            continue;
        }
        if (op == VAR || p.nk[i] == 0) continue;
        const double *x0 = V + (size_t)p.k0[i] * RB;
        const double *x1 = V + (size_t)p.k1[i] * RB;
        const double *fx = V + (size_t)i * RB;
        double *d0 = A + (size_t)p.k0[i] * RB;
        double *d1 = A + (size_t)p.k1[i] * RB;
        double *d2 = A + (size_t)p.k2[i] * RB;
#define ROWS for (int r = 0; r < nb; ++r) if (const double a = ad[r]; a != 0.0)
        switch (op) {
            case NEG: ROWS d0[r] += -a; break;
            case EXP: /* the forward value is exp(x) unless x > 700 */
                ROWS d0[r] += a * (x0[r] > 700.0 ? std::exp(x0[r]) : fx[r]);
                break;
            case LOG: ROWS d0[r] += a / x0[r]; break;
            case ABS: ROWS d0[r] += a * (x0[r] >= 0.0 ? 1.0 : -1.0); break;
            case SQRT: ROWS d0[r] += a / (2.0 * fx[r]); break;
            case SIN: ROWS d0[r] += a * std::cos(x0[r]); break;
            case COS: ROWS d0[r] += -a * std::sin(x0[r]); break;
            case TAN:
                ROWS {
                    const double t = std::cos(x0[r]);
                    d0[r] += a / (t * t);
                }
                break;
            case SINH: ROWS d0[r] += a * std::cosh(x0[r]); break;
            case COSH: ROWS d0[r] += a * std::sinh(x0[r]); break;
            case TANH:
                ROWS {
                    const double t = fx[r];
                    d0[r] += a * (1.0 - t * t);
                }
                break;
            case SIG:
                ROWS {
                    const double s = fx[r];
                    d0[r] += a * s * (1.0 - s);
                }
                break;
            case GAUSS: ROWS d0[r] += a * (-2.0 * x0[r]) * fx[r]; break;
            case SQUARE: ROWS d0[r] += a * 2.0 * x0[r]; break;
            case CUBE: ROWS d0[r] += a * 3.0 * x0[r] * x0[r]; break;
            case ERF: ROWS d0[r] += a * 2.0 * INV_SQRT_PI * std::exp(-x0[r] * x0[r]); break;
            case ERFC: ROWS d0[r] += -a * 2.0 * INV_SQRT_PI * std::exp(-x0[r] * x0[r]); break;
            case ASINH: ROWS d0[r] += a / std::sqrt(x0[r] * x0[r] + 1.0); break;
            case ACOSH:
                ROWS if (x0[r] > 1.0) d0[r] += a / std::sqrt(x0[r] * x0[r] - 1.0);
                break;
            case ATANH:
                ROWS if (std::fabs(x0[r]) < 1.0) d0[r] += a / (1.0 - x0[r] * x0[r]);
                break;
            case ADD:
                ROWS {
                    d0[r] += a;
                    d1[r] += a;
                }
                break;
            case SUB:
                ROWS {
                    d0[r] += a;
                    d1[r] += -a;
                }
                break;
            case MUL:
                ROWS {
                    d0[r] += a * x1[r];
                    d1[r] += a * x0[r];
                }
                break;
            case DIV:
                ROWS {
                    const double q = x1[r];
                    d0[r] += a / q;
                    d1[r] += -a * x0[r] / (q * q);
                }
                break;
            case POW:
                ROWS if (x0[r] > 0.0) {
                    d0[r] += a * x1[r] * std::pow(x0[r], x1[r] - 1.0);
                    d1[r] += a * fx[r] * std::log(x0[r]);
                }
                break;
            case MOD:
                ROWS if (std::fabs(x1[r]) >= 1e-12) {
                    d0[r] += a;
                    d1[r] += -a * std::floor(x0[r] / x1[r]);
                }
                break;
            case MIN:
                ROWS {
                    if (x0[r] < x1[r]) d0[r] += a;
                    else if (x1[r] < x0[r]) d1[r] += a;
                    else {
                        d0[r] += 0.5 * a;
                        d1[r] += 0.5 * a;
                    }
                }
                break;
            case MAX:
                ROWS {
                    if (x0[r] > x1[r]) d0[r] += a;
                    else if (x1[r] > x0[r]) d1[r] += a;
                    else {
                        d0[r] += 0.5 * a;
                        d1[r] += 0.5 * a;
                    }
                }
                break;
            case ATAN2:
                ROWS {
                    const double yy = x0[r], xx = x1[r];
                    const double q = xx * xx + yy * yy;
                    if (q > 0.0) {
                        d0[r] += a * xx / q;
                        d1[r] += -a * yy / q;
                    }
                }
                break;
            case IF:
                ROWS {
                    if (x0[r] > 0.0) d1[r] += a;
                    else d2[r] += a;
                }
                break;
            case AND:
                ROWS {
                    d0[r] += a * indicator(x1[r]);
                    d1[r] += a * indicator(x0[r]);
                }
                break;
            case OR:
                ROWS {
                    d0[r] += a * (1.0 - indicator(x1[r]));
                    d1[r] += a * (1.0 - indicator(x0[r]));
                }
                break;
            case XOR:
                ROWS {
                    d0[r] += a * (1.0 - 2.0 * indicator(x1[r]));
                    d1[r] += a * (1.0 - 2.0 * indicator(x0[r]));
                }
                break;
            default: break; /* step, floor, ceil, round, sign, comparisons, not */
        }
#undef ROWS
    }
}

/* ---- the LM arm (fit.rs:1686-1827, :2318-2336, :2534-2624) ------------------ */

/* One thread's sweep buffers. */
struct Work {
    std::vector<double> V, A, G;
    explicit Work(const Prog &p)
        : V((size_t)std::max(p.size(), 1) * RB), A((size_t)std::max(p.size(), 1) * RB),
          G((size_t)std::max((int)p.cpos.size(), 1) * RB)
    {
    }
};

/* Rows per chunk of a pass that runs on several threads. */
constexpr int64_t CH = 256 * RB;

/* The threads one refit runs on: a Work per thread, the refit's subtree
   cache, and with more than one thread the chunk buffer of weighted
   residuals (and Jacobian rows, [row][k + 1]) plus per-block failure flags.
   A pass on several threads computes rows block-parallel and then takes
   every sum in row order on the calling thread, so the bits do not depend
   on the thread count. */
struct Team {
    int nt = 1;
    std::vector<Work> wk;
    Plan plan;
    bool planned = false;
    std::vector<double> rows;
    std::vector<char> bad;
    Team(const Prog &p, int threads) : nt(std::max(threads, 1))
    {
        wk.reserve(nt);
        for (int t = 0; t < nt; ++t) wk.emplace_back(p);
        if (nt > 1) {
            rows.assign((size_t)CH * (size_t)(p.cpos.size() + 1), 0.0);
            bad.assign((size_t)(CH / RB), 0);
        }
    }
    const Plan *flat_plan() const { return planned ? &plan : nullptr; }
};

inline int thread_index() { return omp_get_thread_num(); }

bool transcendental(int op)
{
    switch (op) {
        case SIN: case COS: case TAN: case EXP: case LOG: case SQRT: case TANH: case SIG:
        case GAUSS: case POW: case SINH: case COSH: case ERF: case ERFC: case ATAN2: case MOD:
        case ASINH: case ACOSH: case ATANH: return true;
        default: return false;
    }
}

/* Cache the values of the largest constant-free subtrees (those whose parent
   holds a constant) over all rows, once per refit, within `cap` bytes: the
   LM re-evaluates the tree dozens of times and these values never change.
   Subtrees are taken by evaluation cost (a library function counts 8, other
   interior nodes 1). A subtree occupies the post-order range ending at its
   root. */
void plan_cache(const Prog &p, const Data &d, size_t cap, Team &tm)
{
    const int m = p.size();
    tm.planned = false;
    if (d.n == 0 || p.cpos.empty()) return;
    std::vector<int> parent(m, -1), span(m, 1), cost(m, 0);
    for (int i = 0; i < m; ++i) {
        const int kids[3] = {p.k0[i], p.k1[i], p.k2[i]};
        cost[i] = p.nk[i] == 0 ? 0 : (transcendental(p.op[i]) ? 8 : 1);
        for (int j = 0; j < p.nk[i]; ++j) {
            parent[kids[j]] = i;
            span[i] += span[kids[j]];
            cost[i] += cost[kids[j]];
        }
    }
    std::vector<int> front;
    for (int i = 0; i < m; ++i)
        if (!p.live[i] && p.nk[i] > 0 && parent[i] >= 0 && p.live[parent[i]]) front.push_back(i);
    std::stable_sort(front.begin(), front.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    const size_t fit = cap / (sizeof(double) * (size_t)d.n);
    if (front.size() > fit) front.resize(fit);
    if (front.empty()) return;
    Plan &pl = tm.plan;
    /* fill: evaluate only the chosen subtrees, block by block */
    Plan fill;
    fill.mode.assign(m, NODE_SKIP);
    pl.mode.assign(m, NODE_EVAL);
    pl.col.assign(m, -1);
    for (size_t f = 0; f < front.size(); ++f) {
        const int r = front[f];
        for (int i = r - span[r] + 1; i < r; ++i) {
            fill.mode[i] = NODE_EVAL;
            pl.mode[i] = NODE_SKIP;
        }
        fill.mode[r] = NODE_EVAL;
        pl.mode[r] = NODE_CACHED;
        pl.col[r] = (int)f;
    }
    pl.cache.assign(front.size() * (size_t)d.n, 0.0);
    const int64_t nblk = (d.n + RB - 1) / RB;
#pragma omp parallel for num_threads(tm.nt) schedule(static) if (tm.nt > 1)
    for (int64_t b = 0; b < nblk; ++b) {
        Work &wk = tm.wk[tm.nt > 1 ? thread_index() : 0];
        const int64_t r0 = b * RB;
        const int nb = (int)std::min<int64_t>(RB, d.n - r0);
        forward<false>(p, d, r0, nb, nullptr, wk.V.data(), &fill);
        for (size_t f = 0; f < front.size(); ++f)
            std::memcpy(pl.cache.data() + f * (size_t)d.n + r0,
                        wk.V.data() + (size_t)front[f] * RB, sizeof(double) * (size_t)nb);
    }
    tm.planned = true;
}

/* Weighted SSE at constants c (fit.rs:1732-1762): +inf on the first
   non-finite weighted residual. */
double sse(const Prog &p, const Data &d, const double *w, const double *c, Team &tm)
{
    double s = 0.0;
    if (tm.nt == 1) {
        Work &wk = tm.wk[0];
        const double *root = wk.V.data() + (size_t)p.root * RB;
        for (int64_t r0 = 0; r0 < d.n; r0 += RB) {
            const int nb = (int)std::min<int64_t>(RB, d.n - r0);
            forward<false>(p, d, r0, nb, c, wk.V.data(), tm.flat_plan());
            for (int r = 0; r < nb; ++r) {
                const double sw = w ? w[r0 + r] : 1.0;
                if (sw == 0.0) continue;
                const double res = std::sqrt(sw) * (root[r] - d.y[r0 + r]);
                if (!std::isfinite(res)) return INF;
                s += res * res;
            }
        }
        return s;
    }
    double *R = tm.rows.data();
    for (int64_t c0 = 0; c0 < d.n; c0 += CH) {
        const int64_t nc = std::min<int64_t>(CH, d.n - c0);
        const int nblk = (int)((nc + RB - 1) / RB);
#pragma omp parallel for num_threads(tm.nt) schedule(static)
        for (int b = 0; b < nblk; ++b) {
            Work &wk = tm.wk[thread_index()];
            const int64_t r0 = c0 + (int64_t)b * RB;
            const int nb = (int)std::min<int64_t>(RB, d.n - r0);
            forward<false>(p, d, r0, nb, c, wk.V.data(), tm.flat_plan());
            const double *root = wk.V.data() + (size_t)p.root * RB;
            char fail = 0;
            for (int r = 0; r < nb; ++r) {
                const double sw = w ? w[r0 + r] : 1.0;
                double res = 0.0;
                if (sw != 0.0) {
                    res = std::sqrt(sw) * (root[r] - d.y[r0 + r]);
                    if (!std::isfinite(res)) fail = 1;
                }
                R[r0 - c0 + r] = res;
            }
            tm.bad[b] = fail;
        }
        for (int b = 0; b < nblk; ++b)
            if (tm.bad[b]) return INF;
        for (int64_t r = 0; r < nc; ++r) {
            if (w && w[c0 + r] == 0.0) continue;
            s += R[r] * R[r];
        }
    }
    return s;
}

/* One block's rows of J^T W J (lower triangle) and J^T W r, in row order.
   False on a non-finite weighted residual or Jacobian entry. Built for the
   host's widest vector unit; the arithmetic is element-wise, so every
   variant gives the same bits. */
__attribute__((target_clones("avx512f", "avx2", "default")))
bool accumulate(int nb, int k, const double *w, const double *y, const double *pred,
                const double *G, double *jtj, double *jtr)
{
    double gw[64];
    for (int r = 0; r < nb; ++r) {
        const double sw = w ? w[r] : 1.0;
        if (sw == 0.0) continue;
        const double s = std::sqrt(sw);
        const double res = s * (pred[r] - y[r]);
        if (!std::isfinite(res)) return false;
        for (int j = 0; j < k; ++j) {
            gw[j] = s * G[(size_t)j * RB + r];
            if (!std::isfinite(gw[j])) return false;
        }
        for (int i = 0; i < k; ++i) {
            jtr[i] += gw[i] * res;
            double *row = jtj + (size_t)i * k;
            const double gi = gw[i];
            for (int j = 0; j <= i; ++j) row[j] += gi * gw[j];
        }
    }
    return true;
}

/* Rows [i0, i1) of J^T W J and J^T W r over a chunk of weighted rows
   ([row][k + 1]: the Jacobian row, then the residual), in row order. Four
   rows at a time: each accumulator is loaded once, takes the four rows'
   products one after the other (the same additions in the same order as
   row by row) and is stored once. A skipped (zero-weight) row is all zeros
   and adds exact zeros, which leave every accumulator unchanged (none of
   them can be -0). */
__attribute__((target_clones("avx512f", "avx2", "default")))
void accumulate_rows(int64_t nc, int k, int i0, int i1, const double *rows, double *jtj,
                     double *jtr)
{
    const int k1 = k + 1;
    int64_t r = 0;
    for (; r + 4 <= nc; r += 4) {
        const double *g0 = rows + (size_t)r * k1, *g1 = g0 + k1, *g2 = g1 + k1, *g3 = g2 + k1;
        for (int i = i0; i < i1; ++i) {
            double t = jtr[i];
            t += g0[i] * g0[k];
            t += g1[i] * g1[k];
            t += g2[i] * g2[k];
            t += g3[i] * g3[k];
            jtr[i] = t;
            const double a0 = g0[i], a1 = g1[i], a2 = g2[i], a3 = g3[i];
            double *row = jtj + (size_t)i * k;
            for (int j = 0; j <= i; ++j) {
                double v = row[j];
                v += a0 * g0[j];
                v += a1 * g1[j];
                v += a2 * g2[j];
                v += a3 * g3[j];
                row[j] = v;
            }
        }
    }
    for (; r < nc; ++r) {
        const double *g = rows + (size_t)r * k1;
        const double res = g[k];
        for (int i = i0; i < i1; ++i) {
            jtr[i] += g[i] * res;
            double *row = jtj + (size_t)i * k;
            const double gi = g[i];
            for (int j = 0; j <= i; ++j) row[j] += gi * g[j];
        }
    }
}

/* J^T W J (lower triangle, then mirrored) and J^T W r at c, rows in order
   (fit.rs:1774-1827). False on a non-finite residual or Jacobian entry. */
bool normal_equations(const Prog &p, const Data &d, const double *w, const double *c, int k,
                      Team &tm, std::vector<double> &jtj, std::vector<double> &jtr)
{
    jtj.assign((size_t)k * k, 0.0);
    jtr.assign(k, 0.0);
    if (tm.nt == 1) {
        Work &wk = tm.wk[0];
        const double *root = wk.V.data() + (size_t)p.root * RB;
        for (int64_t r0 = 0; r0 < d.n; r0 += RB) {
            const int nb = (int)std::min<int64_t>(RB, d.n - r0);
            forward<false>(p, d, r0, nb, c, wk.V.data(), tm.flat_plan());
            backward(p, nb, wk.V.data(), wk.A.data(), wk.G.data());
            if (!accumulate(nb, k, w ? w + r0 : nullptr, d.y + r0, root, wk.G.data(), jtj.data(),
                            jtr.data()))
                return false;
        }
    } else {
        const int k1 = k + 1;
        double *R = tm.rows.data();
        for (int64_t c0 = 0; c0 < d.n; c0 += CH) {
            const int64_t nc = std::min<int64_t>(CH, d.n - c0);
            const int nblk = (int)((nc + RB - 1) / RB);
#pragma omp parallel for num_threads(tm.nt) schedule(static)
            for (int b = 0; b < nblk; ++b) {
                Work &wk = tm.wk[thread_index()];
                const int64_t r0 = c0 + (int64_t)b * RB;
                const int nb = (int)std::min<int64_t>(RB, d.n - r0);
                forward<false>(p, d, r0, nb, c, wk.V.data(), tm.flat_plan());
                backward(p, nb, wk.V.data(), wk.A.data(), wk.G.data());
                const double *root = wk.V.data() + (size_t)p.root * RB;
                char fail = 0;
                for (int r = 0; r < nb; ++r) {
                    double *g = R + (size_t)(r0 - c0 + r) * k1;
                    const double sw = w ? w[r0 + r] : 1.0;
                    if (sw == 0.0) {
                        for (int j = 0; j < k1; ++j) g[j] = 0.0;
                        continue;
                    }
                    const double sq = std::sqrt(sw);
                    const double res = sq * (root[r] - d.y[r0 + r]);
                    if (!std::isfinite(res)) fail = 1;
                    for (int j = 0; j < k; ++j) {
                        g[j] = sq * wk.G[(size_t)j * RB + r];
                        if (!std::isfinite(g[j])) fail = 1;
                    }
                    g[k] = res;
                }
                tm.bad[b] = fail;
            }
            for (int b = 0; b < nblk; ++b)
                if (tm.bad[b]) return false;
            /* the sums stay on this thread: split across threads, each would
               stream the whole chunk, which costs more than it saves */
            accumulate_rows(nc, k, 0, k, R, jtj.data(), jtr.data());
        }
    }
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < i; ++j) jtj[(size_t)j * k + i] = jtj[(size_t)i * k + j];
    return true;
}

/* (A + lambda diag(A) + 1e-12 I) step = b by Cholesky (fit.rs:1686-1727). */
bool damped_solve(const std::vector<double> &a, const std::vector<double> &b, double lambda, int k,
                  std::vector<double> &step)
{
    std::vector<double> m(a), l((size_t)k * k, 0.0), z(k, 0.0);
    for (int i = 0; i < k; ++i) m[(size_t)i * k + i] = m[(size_t)i * k + i] * (1.0 + lambda) + 1e-12;
    for (int i = 0; i < k; ++i) {
        for (int j = 0; j <= i; ++j) {
            double s = m[(size_t)i * k + j];
            for (int q = 0; q < j; ++q) s -= l[(size_t)i * k + q] * l[(size_t)j * k + q];
            if (i == j) {
                if (s <= 1e-18) return false;
                l[(size_t)i * k + j] = std::sqrt(s);
            } else {
                l[(size_t)i * k + j] = s / l[(size_t)j * k + j];
            }
        }
    }
    for (int i = 0; i < k; ++i) {
        double s = b[i];
        for (int q = 0; q < i; ++q) s -= l[(size_t)i * k + q] * z[q];
        z[i] = s / l[(size_t)i * k + i];
    }
    step.assign(k, 0.0);
    for (int i = k - 1; i >= 0; --i) {
        double s = z[i];
        for (int q = i + 1; q < k; ++q) s -= l[(size_t)q * k + i] * step[q];
        step[i] = s / l[(size_t)i * k + i];
    }
    return true;
}

/* Rust's f64::clamp: a NaN stays NaN. */
inline double clamp_c(double v)
{
    if (v < -1e6) v = -1e6;
    if (v > 1e6) v = 1e6;
    return v;
}

/* One damped Gauss-Newton trial from the cached normal equations
   (fit.rs:2318-2336). */
bool gn_trial(const Prog &p, const Data &d, const double *w, const std::vector<double> &c,
              double lambda, int k, const std::vector<double> &jtj, const std::vector<double> &jtr,
              Team &tm, std::vector<double> &trial, double &tsse)
{
    std::vector<double> rhs(k), step;
    for (int i = 0; i < k; ++i) rhs[i] = -jtr[i];
    if (!damped_solve(jtj, rhs, lambda, k, step)) return false;
    trial.resize(k);
    for (int i = 0; i < k; ++i) trial[i] = clamp_c(c[i] + step[i]);
    tsse = sse(p, d, w, trial.data(), tm);
    return true;
}

/* `fit_lm` (fit.rs:2534-2624): returns the weighted SSE at the best
   constants, which it leaves in c. */
double fit_lm(const Prog &p, const Data &d, const double *w, int iters, std::vector<double> &c,
              Team &tm)
{
    const int k = (int)p.cpos.size();
    if (k == 0 || d.n == 0) return sse(p, d, w, nullptr, tm);
    if (iters == 0) return sse(p, d, w, c.data(), tm);
    std::vector<double> best_c = c, jtj, jtr, trial;
    double best = sse(p, d, w, c.data(), tm);
    double lambda = 1e-3;
    bool have = false;
    for (int it = 0; it < std::max(iters, 1); ++it) {
        if (!have) have = normal_equations(p, d, w, c.data(), k, tm, jtj, jtr);
        if (!have) break;
        double tsse;
        if (!gn_trial(p, d, w, c, lambda, k, jtj, jtr, tm, trial, tsse)) break;
        if (tsse < best) {
            c = trial;
            best = tsse;
            best_c = c;
            lambda = std::max(lambda / 8.0, 1e-12);
            have = false;
            if (best == 0.0) break;
        } else {
            lambda *= 6.0;
            if (lambda > 1e9) break;
        }
    }
    /* the undamped Gauss-Newton polish */
    for (int it = 0; it < 4; ++it) {
        if (best == 0.0) break;
        if (!normal_equations(p, d, w, best_c.data(), k, tm, jtj, jtr)) break;
        double tsse;
        if (!gn_trial(p, d, w, best_c, 0.0, k, jtj, jtr, tm, trial, tsse)) break;
        if (tsse < best) {
            best_c = trial;
            best = tsse;
        } else {
            break;
        }
    }
    c = best_c;
    return best;
}

/* ---- predictions and scores ------------------------------------------------ */

void predict(const Prog &p, const Data &d, const double *c, Team &tm, double *out)
{
    const int64_t nblk = (d.n + RB - 1) / RB;
#pragma omp parallel for num_threads(tm.nt) schedule(static) if (tm.nt > 1)
    for (int64_t b = 0; b < nblk; ++b) {
        Work &wk = tm.wk[tm.nt > 1 ? thread_index() : 0];
        const int64_t r0 = b * RB;
        const int nb = (int)std::min<int64_t>(RB, d.n - r0);
        forward<true>(p, d, r0, nb, c, wk.V.data());
        std::memcpy(out + r0, wk.V.data() + (size_t)p.root * RB, sizeof(double) * (size_t)nb);
    }
}

/* The absolute and log-squashed objectives of `metric_score`
   (metrics.rs:852-900 unweighted, :985-1075 weighted). */
double score(const double *pred, const Data &d, int metric)
{
    const int64_t n = d.n;
    if (n == 0) return INF;
    const bool logsq = metric == MT_LOG_SQUASHED;
    if (!d.w) {
        for (int64_t i = 0; i < n; ++i)
            if (!std::isfinite(pred[i])) return INF;
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            const double e = pred[i] - d.y[i];
            s += logsq ? std::log(1.0 + e * e) : std::fabs(e);
        }
        return s / (double)n;
    }
    double total = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        if (!std::isfinite(d.w[i]) || d.w[i] < 0.0) return INF;
        total += d.w[i];
    }
    if (!(total > 0.0)) return INF;
    for (int64_t i = 0; i < n; ++i)
        if (d.w[i] > 0.0 && !std::isfinite(pred[i])) return INF;
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double e = d.w[i] > 0.0 ? pred[i] - d.y[i] : 0.0;
        s += logsq ? d.w[i] * std::log(1.0 + e * e) : d.w[i] * std::fabs(e);
    }
    return s / total;
}

/* The IRLS arm for absolute / log-squashed (fit.rs:3092-3170): majoriser
   weights from the current residuals, a short weighted LM, kept only while
   the configured objective falls; then one longer weighted LM at the final
   weights, kept if it improves. */
double irls(const Prog &p, const Data &d, int iters, int metric, std::vector<double> &c, Team &tm)
{
    const int64_t n = d.n;
    std::vector<double> pred((size_t)std::max<int64_t>(n, 1)), wts((size_t)std::max<int64_t>(n, 1));
    auto weight_of = [&](double r) {
        if (metric == MT_ABSOLUTE) return 1.0 / std::max(std::fabs(r), 1e-6);
        return 1.0 / (1.0 + r * r);
    };
    auto set_weights = [&]() {
        for (int64_t i = 0; i < n; ++i) {
            const double r = pred[i] - d.y[i];
            const double base = d.w ? d.w[i] : 1.0;
            wts[i] = base > 0.0 ? base * std::max(weight_of(r), 0.0) : 0.0;
        }
    };
    predict(p, d, c.data(), tm, pred.data());
    double best = score(pred.data(), d, metric);
    if (!std::isfinite(best)) return best;
    const int rounds = iters < 1 ? 1 : (iters > 4 ? 4 : iters);
    const int inner = std::max(iters / rounds, 1);
    std::vector<double> trial;
    for (int round = 0; round < rounds; ++round) {
        predict(p, d, c.data(), tm, pred.data());
        for (int64_t i = 0; i < n; ++i)
            if (!std::isfinite(pred[i] - d.y[i])) return best;
        set_weights();
        trial = c;
        fit_lm(p, d, wts.data(), inner, trial, tm);
        predict(p, d, trial.data(), tm, pred.data());
        const double s = score(pred.data(), d, metric);
        if (std::isfinite(s) && s < best) {
            best = s;
            c = trial;
        } else {
            break;
        }
    }
    predict(p, d, c.data(), tm, pred.data());
    bool all = true;
    for (int64_t i = 0; i < n; ++i) all = all && std::isfinite(pred[i]);
    if (all) {
        set_weights();
        trial = c;
        fit_lm(p, d, wts.data(), std::max(iters, 4), trial, tm);
        predict(p, d, trial.data(), tm, pred.data());
        const double s = score(pred.data(), d, metric);
        if (std::isfinite(s) && s < best) {
            best = s;
            c = trial;
        }
    }
    return best;
}

bool covered(int metric)
{
    return metric == MT_SQUARED || metric == MT_AIC || metric == MT_AICC || metric == MT_BIC ||
           metric == MT_ABSOLUTE || metric == MT_LOG_SQUASHED;
}

/* One finalist: `fit_weighted_metric` for the covered metrics. */
double refit_one(const int *ops, double *vals, int nn, const Data &d, int iters, int metric,
                 size_t cache_cap, int threads)
{
    Prog p;
    if (!load(ops, vals, nn, p)) return NaN;
    std::vector<double> c(p.cpos.size());
    for (size_t s = 0; s < c.size(); ++s) c[s] = vals[p.cpos[s]];
    Team tm(p, threads);
    if (iters > 0) plan_cache(p, d, cache_cap, tm);
    const bool lsq = metric != MT_ABSOLUTE && metric != MT_LOG_SQUASHED;
    double r;
    if (lsq) {
        r = fit_lm(p, d, d.w, iters, c, tm);
    } else if (iters == 0) {
        std::vector<double> pred((size_t)std::max<int64_t>(d.n, 1));
        predict(p, d, c.data(), tm, pred.data());
        r = score(pred.data(), d, metric);
    } else {
        r = irls(p, d, iters, metric, c, tm);
    }
    for (size_t s = 0; s < c.size(); ++s) vals[p.cpos[s]] = c[s];
    return r;
}

}  // namespace

extern "C" {

int rch_refit_finalists(const int32_t *ops, double *vals, const int32_t *tree_off, int ntrees,
                        const double *cols, int64_t n, int nvars, const double *y, const double *w,
                        int iters, int metric, int threads, double *loss)
{
    if (ntrees < 0 || n < 0 || nvars < 0 || iters < 0) return -1;
    if (ntrees == 0) return 0;
    if (!ops || !vals || !tree_off || !loss || (n > 0 && (!y || (nvars > 0 && !cols)))) return -1;
    if (!covered(metric)) return -2;
    for (int t = 0; t < ntrees; ++t)
        if (tree_off[t + 1] < tree_off[t]) return -1;
    const Data d{cols, n, nvars, y, w};
    int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    nt = std::max(1, nt);
    /* Teams of `team` threads refit finalists concurrently: with at least as
       many finalists as threads every refit runs on one thread; with fewer,
       each refit splits its passes by rows over its team (its sums stay in
       row order). Few rows do not pay for a team. The bits are the same
       either way. */
    const int team = n >= 16384 ? std::max(1, nt / ntrees) : 1;
    const int teams = std::max(1, std::min(ntrees, nt / team));
    /* the subtree caches of the fits in flight share 2 GiB */
    const size_t cap = std::max<size_t>((size_t)16 << 20, ((size_t)2 << 30) / (size_t)teams);
    /* largest first (nodes x (constants + 1)), so the pool ends together */
    std::vector<int> order(ntrees);
    std::vector<long> work(ntrees);
    for (int t = 0; t < ntrees; ++t) {
        order[t] = t;
        long k = 0;
        for (int i = tree_off[t]; i < tree_off[t + 1]; ++i) k += ops[i] == CONST;
        work[t] = (long)(tree_off[t + 1] - tree_off[t]) * (k + 1);
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
    std::atomic<int> next{0};
    auto worker = [&]() {
        for (int q = next.fetch_add(1); q < ntrees; q = next.fetch_add(1)) {
            const int t = order[q];
            const int b = tree_off[t], e = tree_off[t + 1];
            loss[t] = refit_one(ops + b, vals + b, e - b, d, iters, metric, cap, team);
        }
    };
    if (teams == 1) {
        worker();
    } else {
        std::vector<std::thread> pool;
        pool.reserve(teams);
        for (int i = 0; i < teams; ++i) pool.emplace_back(worker);
        for (std::thread &th : pool) th.join();
    }
    return 0;
}

int rch_soa_eval(const int32_t *ops, const double *vals, int nn, const double *cols, int64_t n,
                 int nvars, double *out)
{
    if (n < 0 || nvars < 0 || (n > 0 && !out)) return -1;
    if (n == 0) return 0;
    Prog p;
    if (!ops || !vals || nn <= 0 || !load(ops, vals, nn, p)) return -1;
    const Data d{cols, n, nvars, nullptr, nullptr};
    Team tm(p, 1);
    predict(p, d, nullptr, tm, out);
    return 0;
}

double rch_soa_sse(const int32_t *ops, const double *vals, int nn, const double *cols, int64_t n,
                   int nvars, const double *y)
{
    if (n < 0 || nvars < 0 || (n > 0 && !y)) return NaN;
    if (n == 0) return 0.0;
    Prog p;
    if (!ops || !vals || nn <= 0 || !load(ops, vals, nn, p)) return NaN;
    const Data d{cols, n, nvars, y, nullptr};
    Work wk(p);
    const double *root = wk.V.data() + (size_t)p.root * RB;
    double acc = 0.0;
    for (int64_t r0 = 0; r0 < n; r0 += RB) {
        const int nb = (int)std::min<int64_t>(RB, n - r0);
        forward<true>(p, d, r0, nb, nullptr, wk.V.data());
        for (int r = 0; r < nb; ++r) {
            if (!std::isfinite(root[r])) return INF;
            const double e = root[r] - y[r0 + r];
            acc += e * e;
        }
    }
    return acc;
}

}  /* extern "C" */
