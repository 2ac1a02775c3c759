/*
 * CPU f64 oracle for the rcsr device hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This file restates, in plain C++17, the reference's
 * exact CPU arithmetic for the path the CUDA library replaces: the tree
 * evaluator, the flat value/adjoint sweeps, the historical Levenberg-Marquardt
 * fitter, the L1/log-squashed IRLS wrapper, the metric reducers, the exact
 * integer rank sums and the implicit |f|/||grad f|| metric. Only the tests,
 * `__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py` may load it,
 * and only as the checker (or the timed CPU baseline); the shipped library
 * never calls it.
 *
 * Build: g++ -O2 -ffp-contract=off -fPIC -shared (see oracle/Makefile). The
 * no-contraction flag mirrors Rust's f64 semantics (no implicit FMA), and the
 * transcendental calls go to glibc libm, which is what Rust's f64 methods call
 * on linux-gnu.
 *
 * Trees arrive as two pre-order arrays (`op[i]`, `val[i]`); an operator's arity
 * follows from its code (see `arity`). Constants carry their f64 value in
 * `val`, inputs their column index. Column data is column-major f64
 * `cols[k * n + row]`, the device layout.
 *
 * Every function cites the reference file:line it follows (paths are relative
 * to the reference project's `my-version/` directory).
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <limits>
#include <vector>

namespace {

const double INF = std::numeric_limits<double>::infinity();
const double NaN = std::numeric_limits<double>::quiet_NaN();

/* Tree operator codes. Codes 0..42 are numerically the device opcodes
   (src/cuda/eval.cu:34-83, src/gpu.rs:29-73); 64..66 are the tree-only inverse
   hyperbolics that src/gpu.rs:320-345 lowers before emission. */
enum Op {
    CONST = 0, VAR = 1, ADD = 2, SUB = 3, MUL = 4, DIV = 5, SIN = 6, COS = 7, TAN = 8,
    EXP = 9, LOG = 10, SQRT = 11, ABS = 12, TANH = 13, SIG = 14, SQUARE = 15, CUBE = 16,
    NEG = 17, GAUSS = 18, STEP = 19, POW = 20, SINH = 21, COSH = 22, FLOOR = 23, CEIL = 24,
    ROUND = 25, MOD = 26, ATAN2 = 27, ERF = 28, ERFC = 29, MIN = 30, MAX = 31, IF = 32,
    SIGN = 33, EQUAL = 34, LESS = 35, LESS_OR_EQUAL = 36, GREATER = 37, GREATER_OR_EQUAL = 38,
    AND = 39, OR = 40, XOR = 41, NOT = 42, ASINH = 64, ACOSH = 65, ATANH = 66
};

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

struct Node {
    int op;
    double val;
    std::vector<Node> kids;
};

bool parse(const int *ops, const double *vals, int n, int &pos, Node &out, int depth)
{
    if (pos >= n || depth > 4096) return false;
    out.op = ops[pos];
    out.val = vals[pos];
    ++pos;
    int a = arity(out.op);
    out.kids.resize(a);
    for (int i = 0; i < a; ++i) {
        if (!parse(ops, vals, n, pos, out.kids[i], depth + 1)) return false;
    }
    return true;
}

bool load_tree(const int *ops, const double *vals, int n, Node &t)
{
    int pos = 0;
    if (!parse(ops, vals, n, pos, t, 0)) return false;
    return pos == n;
}

/* Pre-order write-back of a tree's values (constants move; nothing else). */
void store_tree(const Node &t, double *vals, int &pos)
{
    vals[pos++] = t.val;
    for (const Node &k : t.kids) store_tree(k, vals, pos);
}

/* --- expr.rs:930-1041: the reference's own erf/erfc ----------------------- */
const double ERF_EPS = 1e-15;
const double ERF_FPMIN = 1e-300;

double gcf_half(double x)
{
    const double a = 0.5;
    double b = x + 1.0 - a;
    double c = 1.0 / ERF_FPMIN;
    double d = 1.0 / b;
    double h = d;
    for (int i = 1; i < 300; ++i) {
        double an = -(double)i * ((double)i - a);
        b += 2.0;
        d = an * d + b;
        if (std::fabs(d) < ERF_FPMIN) d = ERF_FPMIN;
        c = b + an / c;
        if (std::fabs(c) < ERF_FPMIN) c = ERF_FPMIN;
        d = 1.0 / d;
        double del = d * c;
        h *= del;
        if (std::fabs(del - 1.0) < ERF_EPS) break;
    }
    return std::exp(-x + a * std::log(x) - 0.5 * std::log(M_PI)) * h;
}

double clamp01(double v) { return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); }

double gammp_half(double x)
{
    if (std::isnan(x)) return NaN;
    if (x <= 0.0) return 0.0;
    if (!std::isfinite(x)) return 1.0;
    if (x < 1.5) {
        const double a = 0.5;
        double ap = a;
        double sum = 1.0 / a;
        double del = sum;
        for (int i = 0; i < 300; ++i) {
            ap += 1.0;
            del *= x / ap;
            sum += del;
            if (std::fabs(del) < std::fabs(sum) * ERF_EPS) break;
        }
        return clamp01(sum * std::exp(-x + a * std::log(x) - 0.5 * std::log(M_PI)));
    }
    return clamp01(1.0 - gcf_half(x));
}

double gammq_half(double x)
{
    if (std::isnan(x)) return NaN;
    if (x <= 0.0) return 1.0;
    if (!std::isfinite(x)) return 0.0;
    if (x < 1.5) return clamp01(1.0 - gammp_half(x));
    return clamp01(gcf_half(x));
}

double r_erf(double x)
{
    if (std::isnan(x)) return NaN;
    double p = gammp_half(x * x);
    return x < 0.0 ? -p : p;
}

double r_erfc(double x)
{
    if (std::isnan(x)) return NaN;
    double q = gammq_half(x * x);
    return x < 0.0 ? 2.0 - q : q;
}

/* Rust std's f64::asinh/acosh/atanh (library/std/src/f64.rs, published
   algorithms), which expr.rs:1181-1200 calls. */
double r_asinh(double x)
{
    double ax = std::fabs(x);
    double ix = 1.0 / ax;
    return std::copysign(std::log1p(ax + ax / (std::hypot(1.0, ix) + ix)), x);
}
double r_acosh(double x)
{
    if (x < 1.0) return NaN;
    return std::log(x + std::sqrt(x - 1.0) * std::sqrt(x + 1.0));
}
double r_atanh(double x) { return 0.5 * std::log1p((2.0 * x) / (1.0 - x)); }

double r_min(double a, double b) { return std::fmin(a, b); }
double r_max(double a, double b) { return std::fmax(a, b); }

double cmpf(double a, double b, int op)
{
    if (std::isnan(a) || std::isnan(b)) return NaN;
    bool r;
    switch (op) {
        case EQUAL: r = a == b; break;
        case LESS: r = a < b; break;
        case LESS_OR_EQUAL: r = a <= b; break;
        case GREATER: r = a > b; break;
        default: r = a >= b; break;
    }
    return r ? 1.0 : 0.0;
}

double logicf(double a, double b, int op)
{
    if (std::isnan(a) || std::isnan(b)) return NaN;
    bool x = a > 0.0, y = b > 0.0, r;
    switch (op) {
        case AND: r = x && y; break;
        case OR: r = x || y; break;
        default: r = x != y; break;
    }
    return r ? 1.0 : 0.0;
}

/* --- expr.rs:1054-1326: `expr::eval` with every domain guard ------------- */
double eval(const Node &n, const double *x, int nx)
{
    auto E = [&](int k) { return eval(n.kids[k], x, nx); };
    switch (n.op) {
        case CONST: return n.val;
        case VAR: {
            long i = (long)n.val;
            return (n.val >= 0 && i < nx) ? x[i] : NaN;
        }
        case NEG: return -E(0);
        case EXP: {
            double a = E(0);
            return a > 700.0 ? INF : std::exp(a);
        }
        case LOG: {
            double a = E(0);
            return a > 0.0 ? std::log(a) : NaN;
        }
        case ABS: return std::fabs(E(0));
        case SQRT: {
            double a = E(0);
            return a >= 0.0 ? std::sqrt(a) : NaN;
        }
        case SIN: return std::sin(E(0));
        case COS: return std::cos(E(0));
        case TAN: {
            double t = std::tan(E(0));
            return std::isfinite(t) ? t : NaN;
        }
        case SINH: return std::sinh(E(0));
        case COSH: return std::cosh(E(0));
        case TANH: return std::tanh(E(0));
        case SIG: {
            double a = E(0);
            return 1.0 / (1.0 + std::exp(-a));
        }
        case STEP: return E(0) > 0.0 ? 1.0 : 0.0;
        case GAUSS: {
            double a = E(0);
            return std::exp(-a * a);
        }
        case SQUARE: {
            double a = E(0);
            return a * a;
        }
        case CUBE: {
            double a = E(0);
            return a * a * a;
        }
        case FLOOR: return std::floor(E(0));
        case CEIL: return std::ceil(E(0));
        case ROUND: return std::round(E(0));
        case SIGN: {
            double a = E(0);
            if (a > 0.0) return 1.0;
            if (a < 0.0) return -1.0;
            if (a == 0.0) return 0.0;
            return NaN;
        }
        case ERF: return r_erf(E(0));
        case ERFC: return r_erfc(E(0));
        case ASINH: return r_asinh(E(0));
        case ACOSH: {
            double a = E(0);
            return a >= 1.0 ? r_acosh(a) : NaN;
        }
        case ATANH: {
            double a = E(0);
            return std::fabs(a) < 1.0 ? r_atanh(a) : NaN;
        }
        case ADD: return E(0) + E(1);
        case SUB: return E(0) - E(1);
        case MUL: return E(0) * E(1);
        case DIV: {
            double b = E(1);
            if (std::fabs(b) < 1e-12) return NaN;
            return E(0) / b;
        }
        case POW: {
            double a = E(0), b = E(1);
            if (a < 0.0 && std::fabs(b - std::round(b)) > 1e-9) return NaN;
            return std::pow(a, b);
        }
        case MOD: {
            double a = E(0), b = E(1);
            if (!std::isfinite(a) || !std::isfinite(b) || std::fabs(b) < 1e-12) return NaN;
            return a - b * std::floor(a / b);
        }
        case MIN: {
            double a = E(0), b = E(1);
            if (std::isnan(a) || std::isnan(b)) return NaN;
            return r_min(a, b);
        }
        case MAX: {
            double a = E(0), b = E(1);
            if (std::isnan(a) || std::isnan(b)) return NaN;
            return r_max(a, b);
        }
        case ATAN2: {
            double y = E(0), xx = E(1);
            if (std::isnan(y) || std::isnan(xx)) return NaN;
            return std::atan2(y, xx);
        }
        case IF: return E(0) > 0.0 ? E(1) : E(2);
        case EQUAL: case LESS: case LESS_OR_EQUAL: case GREATER: case GREATER_OR_EQUAL:
            return cmpf(E(0), E(1), n.op);
        case AND: case OR: case XOR: return logicf(E(0), E(1), n.op);
        case NOT: {
            double a = E(0);
            if (std::isnan(a)) return NaN;
            return a > 0.0 ? 0.0 : 1.0;
        }
        default: return NaN;
    }
}

int count_constants(const Node &n)
{
    int t = n.op == CONST ? 1 : 0;
    for (const Node &k : n.kids) t += count_constants(k);
    return t;
}

/* --- fit.rs:1068-1196: the flattened (post-order) tree ------------------- */
struct Flat {
    std::vector<int> op;
    std::vector<double> val;
    std::vector<int> k0, k1, k2, nk;
    std::vector<int> cslot;
    int root = 0;
    int nconst = 0;
};

int build_flat(const Node &n, Flat &f)
{
    int kids[3] = {0, 0, 0};
    for (size_t i = 0; i < n.kids.size(); ++i) kids[i] = build_flat(n.kids[i], f);
    int slot = -1;
    if (n.op == CONST) slot = f.nconst++;
    f.op.push_back(n.op);
    f.val.push_back(n.val);
    f.k0.push_back(kids[0]);
    f.k1.push_back(kids[1]);
    f.k2.push_back(kids[2]);
    f.nk.push_back((int)n.kids.size());
    f.cslot.push_back(slot);
    return (int)f.op.size() - 1;
}

Flat flatten(const Node &t)
{
    Flat f;
    f.root = build_flat(t, f);
    return f;
}

/* Constants in slot order; for a block-free tree this is the pre-order order
   `write_constants` (fit.rs:2626-2646) visits. */
void write_constants(Node &n, const double *c, int &slot)
{
    if (n.op == CONST) n.val = c[slot++];
    for (Node &k : n.kids) write_constants(k, c, slot);
}

/* fit.rs:1211-1382: `value_of`, the flat evaluator's per-node arithmetic. */
double value_of(const Flat &f, int i, const std::vector<double> &v)
{
    auto A = [&](int j) { return v[j == 0 ? f.k0[i] : (j == 1 ? f.k1[i] : f.k2[i])]; };
    switch (f.op[i]) {
        case CONST: return f.val[i];
        case VAR: return f.val[i];
        case NEG: return -A(0);
        case EXP: {
            double x = A(0);
            return x > 700.0 ? INF : std::exp(x);
        }
        case LOG: return std::log(A(0));
        case ABS: return std::fabs(A(0));
        case SQRT: return std::sqrt(A(0));
        case SIN: return std::sin(A(0));
        case COS: return std::cos(A(0));
        case TAN: return std::tan(A(0));
        case SINH: return std::sinh(A(0));
        case COSH: return std::cosh(A(0));
        case TANH: return std::tanh(A(0));
        case SIG: return 1.0 / (1.0 + std::exp(-A(0)));
        case STEP: return A(0) > 0.0 ? 1.0 : 0.0;
        case GAUSS: {
            double x = A(0);
            return std::exp(-x * x);
        }
        case SQUARE: return A(0) * A(0);
        case CUBE: return A(0) * A(0) * A(0);
        case FLOOR: return std::floor(A(0));
        case CEIL: return std::ceil(A(0));
        case ROUND: return std::round(A(0));
        case SIGN: {
            double x = A(0);
            if (x > 0.0) return 1.0;
            if (x < 0.0) return -1.0;
            if (x == 0.0) return 0.0;
            return NaN;
        }
        case ERF: return r_erf(A(0));
        case ERFC: return r_erfc(A(0));
        case ASINH: return r_asinh(A(0));
        case ACOSH: {
            double x = A(0);
            return x >= 1.0 ? r_acosh(x) : NaN;
        }
        case ATANH: {
            double x = A(0);
            return std::fabs(x) < 1.0 ? r_atanh(x) : NaN;
        }
        case ADD: return A(0) + A(1);
        case SUB: return A(0) - A(1);
        case MUL: return A(0) * A(1);
        case DIV: {
            double b = A(1);
            return std::fabs(b) < 1e-12 ? NaN : A(0) / b;
        }
        case POW: return std::pow(A(0), A(1));
        case MOD: {
            double x = A(0), b = A(1);
            if (!std::isfinite(x) || !std::isfinite(b) || std::fabs(b) < 1e-12) return NaN;
            return x - b * std::floor(x / b);
        }
        case MIN: {
            double x = A(0), y = A(1);
            if (std::isnan(x) || std::isnan(y)) return NaN;
            return r_min(x, y);
        }
        case MAX: {
            double x = A(0), y = A(1);
            if (std::isnan(x) || std::isnan(y)) return NaN;
            return r_max(x, y);
        }
        case ATAN2: return std::atan2(A(0), A(1));
        case IF: return A(0) > 0.0 ? A(1) : A(2);
        case EQUAL: case LESS: case LESS_OR_EQUAL: case GREATER: case GREATER_OR_EQUAL:
            return cmpf(A(0), A(1), f.op[i]);
        case AND: case OR: case XOR: return logicf(A(0), A(1), f.op[i]);
        case NOT: {
            double x = A(0);
            if (std::isnan(x)) return NaN;
            return x > 0.0 ? 0.0 : 1.0;
        }
        default: return NaN;
    }
}

/* Row accessor over column-major data. */
struct Rows {
    const double *cols;
    int n;
    int v;
    double at(int row, int k) const { return cols[(size_t)k * (size_t)n + (size_t)row]; }
};

/* fit.rs:1424-1439: `eval_row`. */
void eval_row(const Flat &f, const Rows &x, int row, const double *c, std::vector<double> &v)
{
    for (size_t i = 0; i < f.op.size(); ++i) {
        if (f.cslot[i] >= 0) {
            v[i] = c[f.cslot[i]];
        } else if (f.op[i] == VAR) {
            long idx = (long)f.val[i];
            v[i] = (f.val[i] >= 0 && idx < x.v) ? x.at(row, (int)idx) : NaN;
        } else {
            v[i] = value_of(f, (int)i, v);
        }
    }
}

/* Same sweep over one explicit row vector (input_gradients, fit.rs:3995). */
void eval_row_vec(const Flat &f, const double *x, int nx, const double *c, std::vector<double> &v)
{
    for (size_t i = 0; i < f.op.size(); ++i) {
        if (f.cslot[i] >= 0) {
            v[i] = c[f.cslot[i]];
        } else if (f.op[i] == VAR) {
            long idx = (long)f.val[i];
            v[i] = (f.val[i] >= 0 && idx < nx) ? x[idx] : NaN;
        } else {
            v[i] = value_of(f, (int)i, v);
        }
    }
}

double ind(double x)
{
    if (std::isnan(x)) return NaN;
    return x > 0.0 ? 1.0 : 0.0;
}

const double INV_SQRT_PI = 0.56418958354775628695;

/* fit.rs:1453-1671: `backward_impl`, the reverse-mode adjoint sweep, seeded at
   the root and accumulated into constant slots and/or input columns. */
void backward_impl(const Flat &f, const std::vector<double> &v, std::vector<double> &adj,
                   double *cg, int ncg, double *ig, int nig)
{
    std::fill(adj.begin(), adj.end(), 0.0);
    if (cg) std::fill(cg, cg + ncg, 0.0);
    if (ig) std::fill(ig, ig + nig, 0.0);
    adj[f.root] = 1.0;
    for (int i = (int)f.op.size() - 1; i >= 0; --i) {
        double a = adj[i];
        if (a == 0.0) continue;
        if (f.op[i] == CONST) {
            if (cg && f.cslot[i] >= 0 && f.cslot[i] < ncg) cg[f.cslot[i]] += a;
            continue;
        }
        if (f.op[i] == VAR) {
            long idx = (long)f.val[i];
            if (ig && f.val[i] >= 0 && idx < nig) ig[idx] += a;
            continue;
        }
        if (f.nk[i] == 0) continue;
        int k0 = f.k0[i], k1 = f.k1[i], k2 = f.k2[i];
        double g0 = v[k0];
        double g1 = f.nk[i] > 1 ? v[k1] : 0.0;
        switch (f.op[i]) {
            case NEG: adj[k0] += -a; break;
            case EXP: adj[k0] += a * std::exp(g0); break;
            case LOG: adj[k0] += a / g0; break;
            case ABS: adj[k0] += a * (g0 >= 0.0 ? 1.0 : -1.0); break;
            case SQRT: adj[k0] += a / (2.0 * std::sqrt(g0)); break;
            case SIN: adj[k0] += a * std::cos(g0); break;
            case COS: adj[k0] += -a * std::sin(g0); break;
            case TAN: {
                double t = std::cos(g0);
                adj[k0] += a / (t * t);
            } break;
            case SINH: adj[k0] += a * std::cosh(g0); break;
            case COSH: adj[k0] += a * std::sinh(g0); break;
            case TANH: {
                double t = std::tanh(g0);
                adj[k0] += a * (1.0 - t * t);
            } break;
            case SIG: {
                double s = 1.0 / (1.0 + std::exp(-g0));
                adj[k0] += a * s * (1.0 - s);
            } break;
            case STEP: break;
            case GAUSS: adj[k0] += a * (-2.0 * g0) * std::exp(-g0 * g0); break;
            case SQUARE: adj[k0] += a * 2.0 * g0; break;
            case CUBE: adj[k0] += a * 3.0 * g0 * g0; break;
            case FLOOR: case CEIL: case ROUND: case SIGN: break;
            case ERF: adj[k0] += a * 2.0 * INV_SQRT_PI * std::exp(-g0 * g0); break;
            case ERFC: adj[k0] += -a * 2.0 * INV_SQRT_PI * std::exp(-g0 * g0); break;
            case ASINH: adj[k0] += a / std::sqrt(g0 * g0 + 1.0); break;
            case ACOSH:
                if (g0 > 1.0) adj[k0] += a / std::sqrt(g0 * g0 - 1.0);
                break;
            case ATANH:
                if (std::fabs(g0) < 1.0) adj[k0] += a / (1.0 - g0 * g0);
                break;
            case ADD:
                adj[k0] += a;
                adj[k1] += a;
                break;
            case SUB:
                adj[k0] += a;
                adj[k1] += -a;
                break;
            case MUL:
                adj[k0] += a * g1;
                adj[k1] += a * g0;
                break;
            case DIV: {
                double d = g1;
                adj[k0] += a / d;
                adj[k1] += -a * g0 / (d * d);
            } break;
            case POW:
                if (g0 > 0.0) {
                    adj[k0] += a * g1 * std::pow(g0, g1 - 1.0);
                    adj[k1] += a * std::pow(g0, g1) * std::log(g0);
                }
                break;
            case MOD:
                if (std::fabs(g1) >= 1e-12) {
                    adj[k0] += a;
                    adj[k1] += -a * std::floor(g0 / g1);
                }
                break;
            case MIN:
                if (g0 < g1) adj[k0] += a;
                else if (g1 < g0) adj[k1] += a;
                else {
                    adj[k0] += 0.5 * a;
                    adj[k1] += 0.5 * a;
                }
                break;
            case MAX:
                if (g0 > g1) adj[k0] += a;
                else if (g1 > g0) adj[k1] += a;
                else {
                    adj[k0] += 0.5 * a;
                    adj[k1] += 0.5 * a;
                }
                break;
            case ATAN2: {
                double y = g0, x = g1;
                double d = x * x + y * y;
                if (d > 0.0) {
                    adj[k0] += a * x / d;
                    adj[k1] += -a * y / d;
                }
            } break;
            case IF:
                if (g0 > 0.0) adj[k1] += a;
                else adj[k2] += a;
                break;
            case EQUAL: case LESS: case LESS_OR_EQUAL: case GREATER: case GREATER_OR_EQUAL:
            case NOT: break;
            case AND:
                adj[k0] += a * ind(g1);
                adj[k1] += a * ind(g0);
                break;
            case OR:
                adj[k0] += a * (1.0 - ind(g1));
                adj[k1] += a * (1.0 - ind(g0));
                break;
            case XOR:
                adj[k0] += a * (1.0 - 2.0 * ind(g1));
                adj[k1] += a * (1.0 - 2.0 * ind(g0));
                break;
            default: break;
        }
    }
}

/* fit.rs:1686-1727: damped Cholesky, `(A + lambda diag A + 1e-12 I) d = b`. */
bool solve(const std::vector<std::vector<double>> &a, const std::vector<double> &b, double lambda,
           int k, std::vector<double> &d)
{
    std::vector<std::vector<double>> m = a;
    for (int i = 0; i < k; ++i) m[i][i] = m[i][i] * (1.0 + lambda) + 1e-12;
    std::vector<std::vector<double>> l(k, std::vector<double>(k, 0.0));
    for (int i = 0; i < k; ++i) {
        for (int j = 0; j <= i; ++j) {
            double s = m[i][j];
            for (int p = 0; p < j; ++p) s -= l[i][p] * l[j][p];
            if (i == j) {
                if (s <= 1e-18) return false;
                l[i][j] = std::sqrt(s);
            } else {
                l[i][j] = s / l[j][j];
            }
        }
    }
    std::vector<double> y(k, 0.0);
    for (int i = 0; i < k; ++i) {
        double s = b[i];
        for (int p = 0; p < i; ++p) s -= l[i][p] * y[p];
        y[i] = s / l[i][i];
    }
    d.assign(k, 0.0);
    for (int i = k - 1; i >= 0; --i) {
        double s = y[i];
        for (int p = i + 1; p < k; ++p) s -= l[p][i] * d[p];
        d[i] = s / l[i][i];
    }
    return true;
}

/* fit.rs:1732-1762: weighted SSE; any non-finite residual is +inf. */
double sse(const Flat &f, const Rows &x, const double *y, const double *w, const double *c,
           std::vector<double> &v)
{
    double s = 0.0;
    for (int i = 0; i < x.n; ++i) {
        double sw = w ? w[i] : 1.0;
        if (sw == 0.0) continue;
        eval_row(f, x, i, c, v);
        double r = std::sqrt(sw) * (v[f.root] - y[i]);
        if (!std::isfinite(r)) return INF;
        s += r * r;
    }
    return s;
}

struct Normal {
    std::vector<std::vector<double>> jtj;
    std::vector<double> jtr;
};

/* fit.rs:1774-1827: `normal_equations` (JᵀWJ, JᵀWr), lower triangle in row
   order, mirrored afterwards. */
bool normal_equations(const Flat &f, const Rows &x, const double *y, const double *w,
                      const double *c, int k, std::vector<double> &v, std::vector<double> &adj,
                      std::vector<double> &grad, Normal &out)
{
    out.jtj.assign(k, std::vector<double>(k, 0.0));
    out.jtr.assign(k, 0.0);
    for (int row = 0; row < x.n; ++row) {
        double sw = w ? w[row] : 1.0;
        if (sw == 0.0) continue;
        eval_row(f, x, row, c, v);
        double r = std::sqrt(sw) * (v[f.root] - y[row]);
        if (!std::isfinite(r)) return false;
        backward_impl(f, v, adj, grad.data(), k, nullptr, 0);
        double jw = std::sqrt(sw);
        for (int i = 0; i < k; ++i) {
            double gi = jw * grad[i];
            if (!std::isfinite(gi)) return false;
            out.jtr[i] += gi * r;
            for (int j = 0; j <= i; ++j) out.jtj[i][j] += gi * (jw * grad[j]);
        }
    }
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < i; ++j) out.jtj[j][i] = out.jtj[i][j];
    return true;
}

/* fit.rs:2318-2336: `gn_trial`. */
bool gn_trial(const Flat &f, const Rows &x, const double *y, const double *w,
              const std::vector<double> &c, double lambda, int k, const Normal &ne,
              std::vector<double> &v, std::vector<double> &trial, double &tsse)
{
    std::vector<double> rhs(k);
    for (int i = 0; i < k; ++i) rhs[i] = -ne.jtr[i];
    std::vector<double> step;
    if (!solve(ne.jtj, rhs, lambda, k, step)) return false;
    trial.resize(k);
    for (int i = 0; i < k; ++i) {
        /* Rust's f64::clamp: a NaN stays NaN */
        double t = c[i] + step[i];
        if (t < -1e6) t = -1e6;
        if (t > 1e6) t = 1e6;
        trial[i] = t;
    }
    tsse = sse(f, x, y, w, trial.data(), v);
    return true;
}

/* How the LM loop of `fit_lm` ended, for comparing the device's status
   labels with the CPU's (the reference's CPU fit returns no status; this
   records which of its `break`s was taken). */
struct LmTrace {
    int stop = 0;      /* 0 iterations / lambda / zero loss; 1 solve failed; 2 normal
                          equations not finite */
    int improved = 0;  /* an accepted step (LM or polish) */
    int start_ok = 1;  /* the starting loss was finite */
};

/* fit.rs:2534-2624: `fit_lm`, the historical LM arm. */
double fit_lm(Node &tree, const Rows &x, const double *y, const double *w, int iters,
              LmTrace *trace = nullptr)
{
    Flat f = flatten(tree);
    int k = f.nconst;
    size_t m = f.op.size();
    std::vector<double> v(std::max<size_t>(m, 1)), adj(m), grad(k);
    if (k == 0 || x.n == 0) return sse(f, x, y, w, nullptr, v);
    std::vector<double> c(k);
    for (size_t i = 0; i < m; ++i)
        if (f.cslot[i] >= 0) c[f.cslot[i]] = f.val[i];
    std::vector<double> best_c = c;
    if (iters == 0) return sse(f, x, y, w, c.data(), v);
    double best_sse = sse(f, x, y, w, c.data(), v);
    if (trace) trace->start_ok = std::isfinite(best_sse) ? 1 : 0;
    double lambda = 1e-3;
    bool have = false;
    Normal ne;
    int outer = iters < 1 ? 1 : iters;
    for (int it = 0; it < outer; ++it) {
        if (!have) {
            have = normal_equations(f, x, y, w, c.data(), k, v, adj, grad, ne);
        }
        if (!have) {
            if (trace) trace->stop = 2;
            break;
        }
        std::vector<double> trial;
        double tsse;
        if (!gn_trial(f, x, y, w, c, lambda, k, ne, v, trial, tsse)) {
            if (trace) trace->stop = 1;
            break;
        }
        if (tsse < best_sse) {
            if (trace) trace->improved = 1;
            c = trial;
            best_sse = tsse;
            best_c = c;
            lambda = std::max(lambda / 8.0, 1e-12);
            have = false;
            if (best_sse == 0.0) break;
        } else {
            lambda *= 6.0;
            if (lambda > 1e9) break;
        }
    }
    for (int it = 0; it < 4; ++it) {
        if (best_sse == 0.0) break;
        Normal n2;
        if (!normal_equations(f, x, y, w, best_c.data(), k, v, adj, grad, n2)) break;
        std::vector<double> trial;
        double tsse;
        if (!gn_trial(f, x, y, w, best_c, 0.0, k, n2, v, trial, tsse)) break;
        if (tsse < best_sse) {
            if (trace) trace->improved = 1;
            best_c = trial;
            best_sse = tsse;
        } else {
            break;
        }
    }
    int slot = 0;
    write_constants(tree, best_c.data(), slot);
    return best_sse;
}

/* --- metrics.rs ---------------------------------------------------------- */
enum Metric {
    M_SQUARED = 0, M_ABSOLUTE = 1, M_LOG_SQUASHED = 2, M_SIGNED = 3, M_MAXIMUM = 4,
    M_CORRELATION = 5, M_CORRELATION_SIGNED = 6, M_AIC = 7, M_AICC = 8, M_BIC = 9,
    M_MEDIAN = 15, M_INTERQUARTILE = 16,
    M_RANK_CORRELATION = 20, M_RANK_CORRELATION_SIGNED = 21
};

/* metrics.rs:1128-1154. */
double loglik(int n, double rss) { return rss <= 0.0 ? -INF : (double)n * std::log(rss / (double)n); }
double aic_v(int n, double rss, int k) { return loglik(n, rss) + 2.0 * k; }
double aicc_v(int n, double rss, int k)
{
    double base = loglik(n, rss);
    if (!std::isfinite(base)) return base;
    double denom = (double)n - (double)k - 1.0;
    if (denom <= 0.0) return INF;
    return base + 2.0 * k + 2.0 * k * (k + 1.0) / denom;
}
double bic_v(int n, double rss, int k) { return loglik(n, rss) + (double)k * std::log((double)n); }

/* metrics.rs:1436-1461: Pearson correlation (two-pass, centred). */
double correlation(const double *a, const double *b, int n)
{
    if (n == 0) return 0.0;
    double dn = (double)n, ma = 0.0, mb = 0.0;
    for (int i = 0; i < n; ++i) ma += a[i];
    for (int i = 0; i < n; ++i) mb += b[i];
    ma /= dn;
    mb /= dn;
    double sab = 0.0, sa = 0.0, sb = 0.0;
    for (int i = 0; i < n; ++i) {
        double da = a[i] - ma, db = b[i] - mb;
        sab += da * db;
        sa += da * da;
        sb += db * db;
    }
    if (sa <= 0.0 || sb <= 0.0) return 0.0;
    return sab / (std::sqrt(sa) * std::sqrt(sb));
}

/* metrics.rs:1269-1292: twice the centred average rank. */
bool centred_ranks_doubled(const double *v, int n, std::vector<int64_t> &a)
{
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) return false;
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int p, int q) { return v[p] < v[q]; });
    a.assign(n, 0);
    int i = 0;
    while (i < n) {
        int j = i + 1;
        while (j < n && v[idx[j]] == v[idx[i]]) ++j;
        int64_t centred = (int64_t)(i + j) - (int64_t)n;
        for (int q = i; q < j; ++q) a[idx[q]] = centred;
        i = j;
    }
    return true;
}

struct RankSums {
    __int128 ab = 0, aa = 0, bb = 0;
};

/* metrics.rs:1359-1416: `RankTarget::new` + `sums`. */
bool rank_sums(const double *pred, const double *y, int n, RankSums &s)
{
    std::vector<int64_t> a, b;
    if (!centred_ranks_doubled(y, n, b)) return false;
    if (!centred_ranks_doubled(pred, n, a)) return false;
    for (int i = 0; i < n; ++i) {
        __int128 x = a[i], t = b[i];
        s.ab += x * t;
        s.aa += x * x;
        s.bb += t * t;
    }
    return true;
}

/* metrics.rs:1422-1439 + the `RankSums::correlation` rule (:1326-1336). */
double score_rank_sums(bool ok, const RankSums &s, bool signed_)
{
    if (!ok) return INF;
    if (s.aa == 0 && s.bb == 0 && s.ab == 0) return 1.0;
    double rho = 0.0;
    if (s.aa > 0 && s.bb > 0) rho = (double)s.ab / std::sqrt((double)s.aa * (double)s.bb);
    return signed_ ? 1.0 - rho : 1.0 - std::fabs(rho);
}

double median_abs(std::vector<double> r)
{
    if (r.empty()) return 0.0;
    for (double &e : r) e = std::fabs(e);
    std::sort(r.begin(), r.end());
    size_t n = r.size();
    return n % 2 == 1 ? r[n / 2] : 0.5 * (r[n / 2 - 1] + r[n / 2]);
}

double iq_mean_abs(std::vector<double> r)
{
    if (r.empty()) return 0.0;
    for (double &e : r) e = std::fabs(e);
    std::sort(r.begin(), r.end());
    size_t n = r.size();
    if (n < 4) {
        double s = 0.0;
        for (double e : r) s += e;
        return s / (double)n;
    }
    size_t lo = n / 4, hi = (3 * n) / 4;
    if (hi < lo + 1) hi = lo + 1;
    double s = 0.0;
    for (size_t i = lo; i < hi; ++i) s += r[i];
    return s / (double)(hi - lo);
}

/* metrics.rs:852-900: `score_with_constants` (unweighted). */
double score_unweighted(const double *pred, const double *y, int n, int m, int k)
{
    if (n == 0) return INF;
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(pred[i])) return INF;
    std::vector<double> r(n);
    for (int i = 0; i < n; ++i) r[i] = pred[i] - y[i];
    double dn = (double)n;
    switch (m) {
        case M_ABSOLUTE: {
            double s = 0.0;
            for (double e : r) s += std::fabs(e);
            return s / dn;
        }
        case M_SQUARED: {
            double s = 0.0;
            for (double e : r) s += e * e;
            return s / dn;
        }
        case M_CORRELATION: return 1.0 - std::fabs(correlation(pred, y, n));
        case M_CORRELATION_SIGNED: return 1.0 - correlation(pred, y, n);
        case M_MEDIAN: return median_abs(r);
        case M_MAXIMUM: {
            double mx = 0.0;
            for (double e : r) mx = std::fmax(mx, std::fabs(e));
            return mx;
        }
        case M_SIGNED: {
            double s = 0.0;
            for (double e : r) s += e;
            return std::fabs(s / dn);
        }
        case M_LOG_SQUASHED: {
            double s = 0.0;
            for (double e : r) s += std::log(1.0 + e * e);
            return s / dn;
        }
        case M_INTERQUARTILE: return iq_mean_abs(r);
        case M_RANK_CORRELATION: case M_RANK_CORRELATION_SIGNED: {
            RankSums s;
            bool ok = rank_sums(pred, y, n, s);
            return score_rank_sums(ok, s, m == M_RANK_CORRELATION_SIGNED);
        }
        case M_AIC: case M_AICC: case M_BIC: {
            double rss = 0.0;
            for (double e : r) rss += e * e;
            if (m == M_AIC) return aic_v(n, rss, k);
            if (m == M_AICC) return aicc_v(n, rss, k);
            return bic_v(n, rss, k);
        }
        default: return INF;
    }
}

/* --- classification objectives (metrics.rs:1467-1579, :705-763) --------- */
enum {
    M_LOG_LOSS = 10, M_BRIER = 11, M_HINGE_SIGMOID = 12, M_HINGE_ORDINARY = 13,
    M_HINGE_SQUARED = 14
};

/* metrics.rs:1534-1542: the stable logistic. */
double sigmoid_stable(double x)
{
    if (x >= 0.0) return 1.0 / (1.0 + std::exp(-x));
    const double e = std::exp(x);
    return e / (1.0 + e);
}

/* metrics.rs:1547-1550: ln(1 + exp(-u)) as max(-u, 0) + ln_1p(exp(-|u|)). */
double softplus_neg(double u)
{
    const double a = std::fabs(u);
    return std::fmax(-u, 0.0) + std::log1p(std::exp(-a));
}

/* metrics.rs:1553-1579: one row, p the logit, l in {0, 1}. */
double classification_row_loss(double p, double l, int m)
{
    const double t = 2.0 * l - 1.0;
    const double u = t * p;
    switch (m) {
        case M_LOG_LOSS: return softplus_neg(u);
        case M_BRIER: {
            const double d = sigmoid_stable(p) - l;
            return d * d;
        }
        case M_HINGE_SIGMOID: {
            const double sg = 2.0 * sigmoid_stable(p) - 1.0;
            return std::fmax(1.0 - t * sg, 0.0);
        }
        case M_HINGE_ORDINARY: return std::fmax(1.0 - u, 0.0);
        case M_HINGE_SQUARED: {
            const double h = std::fmax(1.0 - u, 0.0);
            return h * h;
        }
        default: return NaN;
    }
}

/* metrics.rs:1467-1475 `binary_labels` (w == NULL) and :1511-1532
   `binary_labels_weighted`: l = [y > (min + max) / 2] over the positive-weight
   rows. Returns false when a positive-weight target is not finite or none
   exists. */
bool binary_labels(const double *y, const double *w, int n, std::vector<double> &l)
{
    double lo = INF, hi = -INF;
    for (int i = 0; i < n; ++i) {
        if (w && !(w[i] > 0.0)) continue;
        if (w && !std::isfinite(y[i])) return false;
        lo = std::fmin(lo, y[i]);
        hi = std::fmax(hi, y[i]);
    }
    if (w && (!std::isfinite(lo) || !std::isfinite(hi))) return false;
    const double mid = 0.5 * (lo + hi);
    l.assign(n, 0.0);
    for (int i = 0; i < n; ++i) l[i] = ((!w || w[i] > 0.0) && y[i] > mid) ? 1.0 : 0.0;
    return true;
}

/* metrics.rs:705-763 `score_native_weighted`, classification branch: the
   weighted mean row loss; `*status` 0 ok, 2 a non-finite prediction (in a
   positive-weight row) or unusable target, 4 all-zero weights, 1 invalid
   weights. */
double score_classification(const double *pred, const double *y, const double *w, int n, int m,
                            int *status)
{
    *status = 1;
    if (n == 0) return INF;
    if (w) {
        double total = 0.0;
        for (int i = 0; i < n; ++i) {
            if (!std::isfinite(w[i]) || w[i] < 0.0) return INF;
            total += w[i];
        }
        if (!(total > 0.0)) {
            *status = 4;
            return INF;
        }
    }
    for (int i = 0; i < n; ++i)
        if ((!w || w[i] > 0.0) && !std::isfinite(pred[i])) {
            *status = 2;
            return INF;
        }
    double denom = 0.0;
    if (w)
        for (int i = 0; i < n; ++i) denom += w[i];
    else
        denom = (double)n;
    std::vector<double> l;
    if (!binary_labels(y, w, n, l)) {
        *status = 2;
        return INF;
    }
    double sum = 0.0;
    for (int i = 0; i < n; ++i)
        if (!w || w[i] > 0.0) sum += (w ? w[i] : 1.0) * classification_row_loss(pred[i], l[i], m);
    *status = 0;
    return sum / denom;
}

/* metrics.rs:985-1075: `score_weighted` (regression block); the
   classification codes go to `score_native_weighted`'s branch. */
double score_weighted(const double *pred, const double *y, const double *w, int n, int m, int k)
{
    if (m >= M_LOG_LOSS && m <= M_HINGE_SQUARED) {
        int st = 0;
        return score_classification(pred, y, w, n, m, &st);
    }
    if (!w) return score_unweighted(pred, y, n, m, k);
    if (n == 0) return INF;
    double total = 0.0;
    for (int i = 0; i < n; ++i) {
        if (!std::isfinite(w[i]) || w[i] < 0.0) return INF;
        total += w[i];
    }
    if (!(total > 0.0)) return INF;
    for (int i = 0; i < n; ++i)
        if (w[i] > 0.0 && !std::isfinite(pred[i])) return INF;
    std::vector<double> r(n);
    for (int i = 0; i < n; ++i) r[i] = w[i] > 0.0 ? pred[i] - y[i] : 0.0;
    double s = 0.0;
    switch (m) {
        case M_ABSOLUTE:
            for (int i = 0; i < n; ++i) s += w[i] * std::fabs(r[i]);
            return s / total;
        case M_SQUARED:
            for (int i = 0; i < n; ++i) s += w[i] * r[i] * r[i];
            return s / total;
        case M_SIGNED:
            for (int i = 0; i < n; ++i) s += w[i] * r[i];
            return std::fabs(s / total);
        case M_LOG_SQUASHED:
            for (int i = 0; i < n; ++i) s += w[i] * std::log(1.0 + r[i] * r[i]);
            return s / total;
        default: return INF;
    }
}

std::vector<double> predictions(const Node &t, const Rows &x)
{
    std::vector<double> p(x.n);
    std::vector<double> row(x.v);
    for (int i = 0; i < x.n; ++i) {
        for (int k = 0; k < x.v; ++k) row[k] = x.at(i, k);
        p[i] = eval(t, row.data(), x.v);
    }
    return p;
}

double metric_score(const Node &t, const Rows &x, const double *y, const double *w, int m)
{
    std::vector<double> p = predictions(t, x);
    return score_weighted(p.data(), y, w, x.n, m, count_constants(t));
}

/* fit.rs:3092-3170: `irls_fit`; weight_of is the L1 majoriser (fit.rs:2969)
   or the log-squashed weight (fit.rs:2972). */
double irls_fit(Node &tree, const Rows &x, const double *y, const double *w, int iters, int m)
{
    auto weight_of = [&](double r) {
        if (m == M_ABSOLUTE) return 1.0 / std::max(std::fabs(r), 1e-6);
        return 1.0 / (1.0 + r * r);
    };
    double best = metric_score(tree, x, y, w, m);
    if (!std::isfinite(best)) return best;
    int rounds = iters < 1 ? 1 : (iters > 4 ? 4 : iters);
    int inner = std::max(iters / rounds, 1);
    std::vector<double> weights(x.n);
    for (int round = 0; round < rounds; ++round) {
        std::vector<double> pred = predictions(tree, x);
        bool finite = true;
        for (int i = 0; i < x.n; ++i) {
            double r = pred[i] - y[i];
            if (!std::isfinite(r)) {
                finite = false;
                break;
            }
            double base = w ? w[i] : 1.0;
            weights[i] = base > 0.0 ? base * std::max(weight_of(r), 0.0) : 0.0;
        }
        if (!finite) return best;
        Node trial = tree;
        fit_lm(trial, x, y, weights.data(), inner);
        double score = metric_score(trial, x, y, w, m);
        if (std::isfinite(score) && score < best) {
            best = score;
            tree = trial;
        } else {
            break;
        }
    }
    std::vector<double> pred = predictions(tree, x);
    bool all = true;
    for (double p : pred)
        if (!std::isfinite(p)) all = false;
    if (all) {
        for (int i = 0; i < x.n; ++i) {
            double r = pred[i] - y[i];
            double base = w ? w[i] : 1.0;
            weights[i] = base > 0.0 ? base * std::max(weight_of(r), 0.0) : 0.0;
        }
        Node trial = tree;
        fit_lm(trial, x, y, weights.data(), std::max(iters, 4));
        double score = metric_score(trial, x, y, w, m);
        if (std::isfinite(score) && score < best) {
            best = score;
            tree = trial;
        }
    }
    return best;
}

/* fit.rs:2937-2974: `fit_weighted_metric`, the arms this path covers. */
double fit_weighted_metric(Node &tree, const Rows &x, const double *y, const double *w, int iters,
                           int m)
{
    bool least_squares = (m == M_SQUARED || m == M_AIC || m == M_AICC || m == M_BIC);
    if (iters == 0) {
        if (least_squares) return fit_lm(tree, x, y, w, 0);
        return metric_score(tree, x, y, w, m);
    }
    if (least_squares) return fit_lm(tree, x, y, w, iters);
    if (m == M_ABSOLUTE || m == M_LOG_SQUASHED) return irls_fit(tree, x, y, w, iters, m);
    return INF;
}

/* --- implicit.rs:68-409 -------------------------------------------------- */

/* fit.rs:3995-4010: `input_gradients`. */
void input_gradients(const Node &t, const double *x, int nx, double *grad)
{
    Flat f = flatten(t);
    size_t m = f.op.size();
    std::vector<double> c(f.nconst);
    for (size_t i = 0; i < m; ++i)
        if (f.cslot[i] >= 0) c[f.cslot[i]] = f.val[i];
    std::vector<double> v(m), adj(m);
    eval_row_vec(f, x, nx, c.data(), v);
    backward_impl(f, v, adj, nullptr, 0, grad, nx);
}

/* implicit.rs:68-93. */
bool signed_distance(const Node &t, const double *row, int nx, double &d)
{
    double fv = eval(t, row, nx);
    if (!std::isfinite(fv)) return false;
    std::vector<double> g(nx);
    input_gradients(t, row, nx, g.data());
    double norm_sq = 0.0;
    for (double gi : g) {
        if (!std::isfinite(gi)) return false;
        norm_sq += gi * gi;
    }
    double norm = std::sqrt(norm_sq);
    if (!(std::isfinite(norm) && norm > 0.0)) return false;
    d = fv / norm;
    return std::isfinite(d);
}

/* implicit.rs:122-152 (implicit_derivative metric). */
double implicit_score(const Node &t, const Rows &x, const double *w)
{
    if (x.n == 0) return INF;
    double total = 0.0, sum = 0.0;
    std::vector<double> row(x.v);
    for (int i = 0; i < x.n; ++i) {
        double wi = w ? w[i] : 1.0;
        if (!std::isfinite(wi) || wi < 0.0) return INF;
        if (wi == 0.0) continue;
        for (int k = 0; k < x.v; ++k) row[k] = x.at(i, k);
        double d;
        if (!signed_distance(t, row.data(), x.v, d)) return INF;
        d = std::fabs(d);
        total += wi;
        sum += wi * d;
    }
    if (!(std::isfinite(total) && total > 0.0)) return INF;
    return sum / total;
}

/* implicit.rs:156-174. */
bool implicit_residuals(const Node &t, const Rows &x, const double *w, std::vector<double> &out)
{
    out.resize(x.n);
    std::vector<double> row(x.v);
    for (int i = 0; i < x.n; ++i) {
        double wi = w ? w[i] : 1.0;
        if (!std::isfinite(wi) || wi < 0.0) return false;
        if (wi == 0.0) {
            out[i] = 0.0;
            continue;
        }
        for (int k = 0; k < x.v; ++k) row[k] = x.at(i, k);
        double d;
        if (!signed_distance(t, row.data(), x.v, d)) return false;
        out[i] = std::sqrt(wi) * d;
    }
    return true;
}

double cost(const std::vector<double> &r)
{
    double s = 0.0;
    for (double v : r) s += v * v;
    return s;
}

/* implicit.rs:215-253: Gaussian elimination with partial pivoting. */
bool gauss_solve(const std::vector<std::vector<double>> &a, const std::vector<double> &b,
                 double lambda, int k, std::vector<double> &d)
{
    std::vector<std::vector<double>> m(k, std::vector<double>(k + 1, 0.0));
    for (int i = 0; i < k; ++i) {
        for (int j = 0; j < k; ++j) m[i][j] = a[i][j];
        m[i][i] = m[i][i] * (1.0 + lambda) + 1e-12;
        m[i][k] = b[i];
    }
    for (int col = 0; col < k; ++col) {
        int piv = col;
        for (int r = col + 1; r < k; ++r)
            if (std::fabs(m[r][col]) > std::fabs(m[piv][col])) piv = r;
        if (std::fabs(m[piv][col]) < 1e-300) return false;
        std::swap(m[col], m[piv]);
        for (int r = col + 1; r < k; ++r) {
            double factor = m[r][col] / m[col][col];
            if (factor != 0.0)
                for (int c = col; c <= k; ++c) m[r][c] -= factor * m[col][c];
        }
    }
    d.assign(k, 0.0);
    for (int i = k - 1; i >= 0; --i) {
        double s = m[i][k];
        for (int j = i + 1; j < k; ++j) s -= m[i][j] * d[j];
        d[i] = s / m[i][i];
    }
    return true;
}

Node with_constants(const Node &base, const std::vector<double> &c)
{
    Node t = base;
    int slot = 0;
    write_constants(t, c.data(), slot);
    return t;
}

void collect_constants(const Node &n, std::vector<double> &out)
{
    if (n.op == CONST) out.push_back(n.val);
    for (const Node &k : n.kids) collect_constants(k, out);
}

double rss_of(const Node &t, const Rows &x, const double *w)
{
    std::vector<double> r;
    if (!implicit_residuals(t, x, w, r)) return INF;
    return cost(r);
}

/* implicit.rs:277-409: LM on the signed geometric residual with a
   central-difference Jacobian. */
double implicit_fit(Node &tree, const Rows &x, const double *w, int iters)
{
    if (x.n == 0) return INF;
    std::vector<double> initial;
    collect_constants(tree, initial);
    int k = (int)initial.size();
    if (k == 0) return rss_of(tree, x, w);
    if (iters == 0) return rss_of(tree, x, w);
    Node base = tree;
    std::vector<double> base_r;
    if (!implicit_residuals(base, x, w, base_r)) return INF;
    std::vector<double> best_c = initial;
    double best_sse = cost(base_r);
    std::vector<double> c = best_c;
    double lambda = 1e-3;
    int n = x.n;
    int outer = iters < 1 ? 1 : iters;
    for (int it = 0; it < outer; ++it) {
        std::vector<double> r;
        if (!implicit_residuals(with_constants(base, c), x, w, r)) break;
        std::vector<std::vector<double>> jac(n, std::vector<double>(k, 0.0));
        bool ok = true;
        for (int j = 0; j < k && ok; ++j) {
            double h = 1e-6 * (1.0 + std::fabs(c[j]));
            std::vector<double> cp = c, cm = c;
            cp[j] += h;
            cm[j] -= h;
            std::vector<double> rp, rm;
            if (implicit_residuals(with_constants(base, cp), x, w, rp) &&
                implicit_residuals(with_constants(base, cm), x, w, rm)) {
                for (int i = 0; i < n; ++i) jac[i][j] = (rp[i] - rm[i]) / (2.0 * h);
            } else {
                ok = false;
            }
        }
        if (!ok) break;
        std::vector<std::vector<double>> jtj(k, std::vector<double>(k, 0.0));
        std::vector<double> jtr(k, 0.0);
        for (int i = 0; i < n && ok; ++i) {
            for (int a = 0; a < k; ++a) {
                double ga = jac[i][a];
                if (!std::isfinite(ga)) {
                    ok = false;
                    break;
                }
                jtr[a] += ga * r[i];
                for (int b = 0; b <= a; ++b) jtj[a][b] += ga * jac[i][b];
            }
        }
        if (!ok) break;
        for (int a = 0; a < k; ++a)
            for (int b = 0; b < a; ++b) jtj[b][a] = jtj[a][b];
        std::vector<double> rhs(k);
        for (int a = 0; a < k; ++a) rhs[a] = -jtr[a];
        std::vector<double> step;
        if (!gauss_solve(jtj, rhs, lambda, k, step)) {
            lambda *= 6.0;
            if (lambda > 1e9) break;
            continue;
        }
        std::vector<double> trial(k);
        for (int a = 0; a < k; ++a) trial[a] = std::min(1e6, std::max(-1e6, c[a] + step[a]));
        std::vector<double> rt;
        if (implicit_residuals(with_constants(base, trial), x, w, rt)) {
            double s = cost(rt);
            if (s < best_sse) {
                best_sse = s;
                best_c = trial;
                c = trial;
                lambda = std::max(lambda / 8.0, 1e-12);
                if (best_sse == 0.0) break;
            } else {
                lambda *= 6.0;
                if (lambda > 1e9) break;
            }
        } else {
            lambda *= 6.0;
            if (lambda > 1e9) break;
        }
    }
    if (best_sse < rss_of(tree, x, w)) {
        int slot = 0;
        write_constants(tree, best_c.data(), slot);
    }
    return best_sse;
}

}  // namespace

/* ------------------------------------------------------------------------ */
/* C ABI for the ctypes test harness. Trees are pre-order (op, val) arrays.  */
/* A function that fits writes the fitted values back into `val`.           */
/* ------------------------------------------------------------------------ */
extern "C" {

int or_tree_ok(const int *op, const double *val, int nn)
{
    Node t;
    return load_tree(op, val, nn, t) ? 1 : 0;
}

/* expr::eval over every row of column-major f64 data. */
int or_predict(const int *op, const double *val, int nn, const double *cols, int n, int v,
               double *out)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return -1;
    Rows x{cols, n, v};
    std::vector<double> p = predictions(t, x);
    std::memcpy(out, p.data(), sizeof(double) * (size_t)n);
    return 0;
}

/* gpu.rs:2900-2917 `cpu_sse`: f32 columns widened to f64, the 1e30 rule. */
double or_cpu_sse(const int *op, const double *val, int nn, const float *cols, int n, int v,
                  const float *y)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return NaN;
    std::vector<double> row(v);
    double s = 0.0;
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < v; ++k) row[k] = (double)cols[(size_t)k * n + i];
        double pred = eval(t, row.data(), v);
        if (!std::isfinite(pred) || std::fabs(pred) > 1e30) {
            s += 1e30;
            continue;
        }
        double r = pred - (double)y[i];
        s += r * r;
    }
    return s;
}

/* metrics::score_weighted on expr::eval predictions; `w` may be NULL. */
double or_score(const int *op, const double *val, int nn, const double *cols, int n, int v,
                const double *y, const double *w, int metric)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return NaN;
    Rows x{cols, n, v};
    return metric_score(t, x, y, w, metric);
}

/* metrics::score_weighted on a given prediction vector. */
double or_score_pred(const double *pred, const double *y, const double *w, int n, int metric, int k)
{
    return score_weighted(pred, y, w, n, metric, k);
}

/* fit::fit_weighted_metric (squared family via fit_lm, absolute/log-squashed
   via irls_fit). Returns the fitted objective; constants are written back. */
double or_fit(const int *op, double *val, int nn, const double *cols, int n, int v, const double *y,
              const double *w, int iters, int metric)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return NaN;
    Rows x{cols, n, v};
    double r = fit_weighted_metric(t, x, y, w, iters, metric);
    int pos = 0;
    store_tree(t, val, pos);
    return r;
}

/* The flat evaluator's weighted SSE at the tree's current constants
   (fit_weighted(tree, .., 0) in the reference tests). */
double or_flat_sse(const int *op, const double *val, int nn, const double *cols, int n, int v,
                   const double *y, const double *w)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return NaN;
    Rows x{cols, n, v};
    return fit_lm(t, x, y, w, 0);
}

/* One row: value (flat evaluator) and the constant/input gradients from
   `backward_impl`. `cg` has nconst entries, `ig` has v entries (either may be
   NULL). Returns the number of constants, or -1. */
int or_row_grad(const int *op, const double *val, int nn, const double *row, int v, double *value,
                double *cg, double *ig)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return -1;
    Flat f = flatten(t);
    size_t m = f.op.size();
    std::vector<double> c(f.nconst);
    for (size_t i = 0; i < m; ++i)
        if (f.cslot[i] >= 0) c[f.cslot[i]] = f.val[i];
    std::vector<double> vv(m), adj(m);
    eval_row_vec(f, row, v, c.data(), vv);
    if (value) *value = vv[f.root];
    std::vector<double> gbuf(f.nconst);
    backward_impl(f, vv, adj, gbuf.data(), f.nconst, ig, ig ? v : 0);
    if (cg) std::memcpy(cg, gbuf.data(), sizeof(double) * gbuf.size());
    return f.nconst;
}

/* implicit::score (implicit_derivative). */
double or_implicit_score(const int *op, const double *val, int nn, const double *cols, int n, int v,
                         const double *w)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return NaN;
    Rows x{cols, n, v};
    return implicit_score(t, x, w);
}

/* implicit::fit; constants are written back. */
double or_implicit_fit(const int *op, double *val, int nn, const double *cols, int n, int v,
                       const double *w, int iters)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return NaN;
    Rows x{cols, n, v};
    double r = implicit_fit(t, x, w, iters);
    int pos = 0;
    store_tree(t, val, pos);
    return r;
}

/* RankTarget::sums: three exact i128 sums as (hi, lo) u64 pairs
   [ab_hi, ab_lo, aa_hi, aa_lo, bb_hi, bb_lo]. Returns 0, or -1 when a value
   is not finite. */
int or_rank_sums(const double *pred, const double *y, int n, uint64_t *out)
{
    RankSums s;
    if (!rank_sums(pred, y, n, s)) return -1;
    __int128 v[3] = {s.ab, s.aa, s.bb};
    for (int i = 0; i < 3; ++i) {
        unsigned __int128 u = (unsigned __int128)v[i];
        out[2 * i] = (uint64_t)(u >> 64);
        out[2 * i + 1] = (uint64_t)u;
    }
    return 0;
}

int or_centred_ranks_doubled(const double *v, int n, int64_t *out)
{
    std::vector<int64_t> a;
    if (!centred_ranks_doubled(v, n, a)) return -1;
    std::memcpy(out, a.data(), sizeof(int64_t) * (size_t)n);
    return 0;
}

/* fit_lm (fit.rs:2534-2624) with how its LM loop ended: label[0] = 0 when it
   ran out of iterations, lambda or loss, 1 when a damped solve failed, 2 when
   the normal equations were not finite; label[1] = an accepted step;
   label[2] = a finite starting loss. Constants are written back. */
double or_fit_lm_traced(const int *op, double *val, int nn, const double *cols, int n, int v,
                        const double *y, const double *w, int iters, int *label)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return NaN;
    Rows x{cols, n, v};
    LmTrace tr;
    double r = fit_lm(t, x, y, w, iters, &tr);
    label[0] = tr.stop;
    label[1] = tr.improved;
    label[2] = tr.start_ok;
    int pos = 0;
    store_tree(t, val, pos);
    return r;
}

/* The tree's constants in the flat evaluator's slot order (fit.rs:1068-1196
   `flatten`, the order proposals and `write_constants` use). Returns the
   count, or -1. */
int or_flat_constants(const int *op, const double *val, int nn, double *out)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return -1;
    Flat f = flatten(t);
    for (size_t i = 0; i < f.op.size(); ++i)
        if (f.cslot[i] >= 0) out[f.cslot[i]] = f.val[i];
    return f.nconst;
}

/* Whether fit.rs's `normal_equations` (fit.rs:1774-1827) are finite at the
   tree's constants: 1 finite, 0 not, -1 for a bad tree. */
int or_normal_equations_ok(const int *op, const double *val, int nn, const double *cols, int n,
                           int v, const double *y, const double *w)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return -1;
    Rows x{cols, n, v};
    Flat f = flatten(t);
    const int k = f.nconst;
    const size_t m = f.op.size();
    std::vector<double> c(k), vv(std::max<size_t>(m, 1)), adj(m), grad(k);
    for (size_t i = 0; i < m; ++i)
        if (f.cslot[i] >= 0) c[f.cslot[i]] = f.val[i];
    Normal ne;
    return normal_equations(f, x, y, w, c.data(), k, vv, adj, grad, ne) ? 1 : 0;
}

/* fit/gpu.rs:245-317 `verify_proposal` for the metrics the device fit
   serves here (squared, absolute, log-squashed; the signed projection and
   the rank family are not restated): apply the proposal to a clone and
   accept it only when it is finite and no worse than the starting constants,
   on the weighted SSE of the flat evaluator for squared (fit.rs `sse`) and on
   the configured objective otherwise. Returns 0 (accepted, the constants are
   written into `val` and `*value` is the proposal's exact objective) or 1
   (rejected, `val` untouched). */
int or_verify_proposal(const int *op, double *val, int nn, const double *cols, int n, int v,
                       const double *y, const double *w, int metric, const double *proposal,
                       int np, double *value)
{
    Node t;
    if (!load_tree(op, val, nn, t)) return 1;
    Rows x{cols, n, v};
    Flat f = flatten(t);
    if (np != f.nconst) return 1;
    for (int i = 0; i < np; ++i)
        if (!std::isfinite(proposal[i])) return 1;
    std::vector<double> c0(f.nconst);
    for (size_t i = 0; i < f.op.size(); ++i)
        if (f.cslot[i] >= 0) c0[f.cslot[i]] = f.val[i];
    Node trial = t;
    int slot = 0;
    write_constants(trial, proposal, slot);
    double start, cand;
    if (metric == M_SQUARED) {
        std::vector<double> vv(std::max<size_t>(f.op.size(), 1));
        start = sse(f, x, y, w, c0.data(), vv);
        cand = sse(f, x, y, w, proposal, vv);
    } else {
        start = metric_score(t, x, y, w, metric);
        cand = metric_score(trial, x, y, w, metric);
    }
    if (!std::isfinite(cand) || !std::isfinite(start) || cand > start) return 1;
    int pos = 0;
    store_tree(trial, val, pos);
    *value = cand;
    return 0;
}

/* fit/gpu.rs:176-213 `fit_batch_verified`, one tree: a missing proposal
   (np < 0: the device status was not usable or a constant not finite) or a
   rejected one falls back on the exact CPU fit from the starting constants
   (`fit_weighted_metric`). Returns the tree's score; *state = 0 device
   answer accepted, 1 rejected (CPU fit), 2 no proposal (CPU fit). */
double or_fit_verified(const int *op, double *val, int nn, const double *cols, int n, int v,
                       const double *y, const double *w, int iters, int metric,
                       const double *proposal, int np, int *state)
{
    double value = NaN;
    if (np >= 0) {
        if (or_verify_proposal(op, val, nn, cols, n, v, y, w, metric, proposal, np, &value) ==
            0) {
            *state = 0;
            return value;
        }
        *state = 1;
    } else {
        *state = 2;
    }
    return or_fit(op, val, nn, cols, n, v, y, w, iters, metric);
}

/* The binary labels a classification objective derives from y
   (metrics.rs:1467-1532): out[i] = 1 or 0. Returns 0, or -1 when the
   weighted rule has no usable target. */
int or_binary_labels(const double *y, const double *w, int n, double *out)
{
    std::vector<double> l;
    if (!binary_labels(y, w, n, l)) return -1;
    std::memcpy(out, l.data(), sizeof(double) * (size_t)n);
    return 0;
}

double or_erf(double x) { return r_erf(x); }
double or_erfc(double x) { return r_erfc(x); }

}  /* extern "C" */
