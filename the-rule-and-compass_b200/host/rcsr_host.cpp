/*
 * Host-side compiler for the device path: expression tree -> device program.
 *
 * This is the caller side of the C ABI, restated in C++ from the reference's
 * Rust host layer:
 *   - `compile_program` (my-version/src/gpu.rs:198-219): `lower` (asinh /
 *     acosh / atanh rewrites, :320-345), the `peak_stack` guard (:952-969,
 *     host limit 56, :127) and `emit` (:349-438) into postfix words;
 *   - `gpu_fit_plan_reason` (my-version/src/fit.rs:985-1056) with `flatten`
 *     (:1068-1196): post-order 4-word records [op, kid0, kid1, slot], the
 *     constants in slot order, the correlation gauge (fit/correlation.rs:
 *     83-128) and the rejection reasons.
 *
 * Trees arrive as pre-order (op, val) arrays; operator codes 0..42 are the
 * device opcodes, 64..66 the inverse hyperbolics. Exposed through a small C
 * API (rch_*) for the Python package and the benchmark.
 */
#include "rcsr_host.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

enum {
    CONST = 0, VAR = 1, ADD = 2, SUB = 3, MUL = 4, DIV = 5, SIN = 6, COS = 7, TAN = 8, EXP = 9,
    LOG = 10, SQRT = 11, ABS = 12, TANH = 13, SIG = 14, SQUARE = 15, CUBE = 16, NEG = 17,
    GAUSS = 18, STEP = 19, POW = 20, SINH = 21, COSH = 22, FLOOR = 23, CEIL = 24, ROUND = 25,
    MOD = 26, ATAN2 = 27, ERF = 28, ERFC = 29, MIN = 30, MAX = 31, IF = 32, SIGN = 33,
    EQUAL = 34, LESS = 35, LESS_OR_EQUAL = 36, GREATER = 37, GREATER_OR_EQUAL = 38, AND = 39,
    OR = 40, XOR = 41, NOT = 42, ASINH = 64, ACOSH = 65, ATANH = 66, HALT = 255
};

const int HOST_MAX_STACK = 56;
const int GPU_FIT_MAX_CONSTANTS = 20;
const int GPU_FIT_MAX_NODES = 96;

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

bool known(int op) { return (op >= 0 && op <= 42) || op == ASINH || op == ACOSH || op == ATANH; }

struct Node {
    int op;
    double val;
    std::vector<Node> kids;
};

Node mk(int op, std::vector<Node> kids) { return Node{op, 0.0, std::move(kids)}; }
Node cst(double v) { return Node{CONST, v, {}}; }

bool parse(const int *ops, const double *vals, int n, int &pos, Node &out, int depth)
{
    if (pos >= n || depth > 4096) return false;
    out.op = ops[pos];
    out.val = vals[pos];
    ++pos;
    if (!known(out.op)) return false;
    out.kids.resize(arity(out.op));
    for (Node &k : out.kids)
        if (!parse(ops, vals, n, pos, k, depth + 1)) return false;
    return true;
}

bool load(const int *ops, const double *vals, int n, Node &t)
{
    int pos = 0;
    return parse(ops, vals, n, pos, t, 0) && pos == n;
}

/* The tree of one postfix program of `len` words (the words `emit` writes
   and the device variation engine builds): [CONST, f32 bits] (the value
   widened to f64), [VAR, index], operator words, up to HALT. False for a
   program that is not one well-formed expression (a truncated operand, an
   unknown or under-supplied operator, no HALT, or not exactly one value). */
bool load_postfix(const uint32_t *w, int len, Node &t)
{
    std::vector<Node> st;
    for (int i = 0; i < len;) {
        const int op = (int)w[i++];
        if (op == HALT) {
            if (st.size() != 1) return false;
            t = std::move(st.back());
            return true;
        }
        if (op == CONST || op == VAR) {
            if (i >= len) return false;
            const uint32_t a = w[i++];
            if (op == CONST) {
                float f;
                memcpy(&f, &a, sizeof f);
                st.push_back(Node{CONST, (double)f, {}});
            } else {
                st.push_back(Node{VAR, (double)a, {}});
            }
            continue;
        }
        const int k = arity(op);
        if (!known(op) || (int)st.size() < k) return false;
        Node n{op, 0.0, {}};
        n.kids.assign(std::make_move_iterator(st.end() - k), std::make_move_iterator(st.end()));
        st.erase(st.end() - k, st.end());
        st.push_back(std::move(n));
    }
    return false;
}

/* gpu.rs:320-345 `lower`. */
Node lower(const Node &n, bool &changed)
{
    if (n.op == CONST || n.op == VAR) return n;
    std::vector<Node> k;
    for (const Node &c : n.kids) k.push_back(lower(c, changed));
    if (n.op == ASINH) {
        changed = true;
        const Node x = k[0];
        Node sgn = mk(SUB, {mk(STEP, {x}), mk(STEP, {mk(NEG, {x})})});
        Node mag = mk(LOG, {mk(ADD, {mk(ABS, {x}), mk(SQRT, {mk(ADD, {mk(MUL, {x, x}), cst(1.0)})})})});
        return mk(MUL, {sgn, mag});
    }
    if (n.op == ACOSH) {
        changed = true;
        const Node x = k[0];
        return mk(LOG, {mk(ADD, {x, mk(SQRT, {mk(MUL, {mk(SUB, {x, cst(1.0)}), mk(ADD, {x, cst(1.0)})})})})});
    }
    if (n.op == ATANH) {
        changed = true;
        const Node x = k[0];
        return mk(MUL, {cst(0.5), mk(LOG, {mk(DIV, {mk(ADD, {cst(1.0), x}), mk(SUB, {cst(1.0), x})})})});
    }
    Node out{n.op, n.val, std::move(k)};
    return out;
}

/* gpu.rs:952-969 `peak_stack`. */
void peak_walk(const Node &n, int &cur, int &peak)
{
    for (const Node &k : n.kids) peak_walk(k, cur, peak);
    const int a = (int)n.kids.size();
    if (a == 0) {
        ++cur;
        if (cur > peak) peak = cur;
    } else if (a > 1) {
        cur -= a - 1;
    }
}

/* gpu.rs:349-438 `emit`. */
bool emit(const Node &n, std::vector<uint32_t> &out)
{
    if (n.op == CONST) {
        out.push_back(CONST);
        float f = (float)n.val;
        uint32_t bits;
        memcpy(&bits, &f, 4);
        out.push_back(bits);
        return true;
    }
    if (n.op == VAR) {
        out.push_back(VAR);
        out.push_back((uint32_t)n.val);
        return true;
    }
    if (n.op == ASINH || n.op == ACOSH || n.op == ATANH) return false;
    for (const Node &k : n.kids)
        if (!emit(k, out)) return false;
    out.push_back((uint32_t)n.op);
    return true;
}

/* fit.rs:1068-1196 `flatten` for block-free trees. */
struct Flat {
    std::vector<int> op, k0, k1, cslot;
    std::vector<double> val;
    int nconst = 0;
};

int build(const Node &n, Flat &f)
{
    int kids[3] = {0, 0, 0};
    for (size_t i = 0; i < n.kids.size(); ++i) kids[i] = build(n.kids[i], f);
    int slot = -1;
    if (n.op == CONST) slot = f.nconst++;
    f.op.push_back(n.op);
    f.val.push_back(n.val);
    f.k0.push_back(kids[0]);
    f.k1.push_back(kids[1]);
    f.cslot.push_back(slot);
    return (int)f.op.size() - 1;
}

/* fit.rs:890-920 `gpu_fit_opcode`. */
bool fit_opcode(int op)
{
    switch (op) {
        case CONST: case VAR: case ADD: case SUB: case MUL: case DIV: case SIN: case COS:
        case TAN: case EXP: case LOG: case SQRT: case ABS: case TANH: case SIG: case SQUARE:
        case CUBE: case NEG: case GAUSS: case POW: case SINH: case COSH: case ERF: case ERFC:
            return true;
        default: return false;
    }
}

/* gpu_fit_plan_reason of a loaded tree (rch_fit_plan's contract). */
int plan_tree(const Node &t, uint32_t *words, int cap, double *c0, int cap_c, int *gauge,
              int *nconst, int allow_no_constants)
{
    Flat f;
    build(t, f);
    const int m = (int)f.op.size();
    if (f.nconst == 0 && !allow_no_constants) return -3;
    if (f.nconst > GPU_FIT_MAX_CONSTANTS) return -1;
    if (m > GPU_FIT_MAX_NODES) return -2;
    for (int i = 0; i < m; ++i)
        if (!fit_opcode(f.op[i])) return -5;
    if (4 * m > cap || f.nconst > cap_c) return -6;
    for (int i = 0; i < m; ++i) {
        uint32_t slot;
        if (f.cslot[i] >= 0) slot = (uint32_t)f.cslot[i];
        else if (f.op[i] == VAR) slot = (uint32_t)f.val[i];
        else slot = 0xFFFFFFFFu;
        const int a = arity(f.op[i]);
        words[4 * i] = (uint32_t)f.op[i];
        words[4 * i + 1] = a >= 1 ? (uint32_t)f.k0[i] : 0u;
        words[4 * i + 2] = a >= 2 ? (uint32_t)f.k1[i] : 0u;
        words[4 * i + 3] = slot;
        if (f.cslot[i] >= 0) c0[f.cslot[i]] = f.val[i];
    }
    /* fit/correlation.rs:83-128 `gauge_of`. */
    gauge[0] = -1;
    gauge[1] = -1;
    const int root = m - 1;
    if (f.op[root] == MUL) {
        const int a = f.k0[root], b = f.k1[root];
        if (f.cslot[a] >= 0 && f.cslot[b] < 0) gauge[0] = f.cslot[a];
        else if (f.cslot[b] >= 0 && f.cslot[a] < 0) gauge[0] = f.cslot[b];
    } else if (f.op[root] == ADD) {
        const int ks[2] = {f.k0[root], f.k1[root]};
        for (int side = 0; side < 2; ++side) {
            const int mm = ks[side], bb = ks[1 - side];
            if (f.op[mm] != MUL || f.cslot[bb] < 0) continue;
            const int x = f.k0[mm], y = f.k1[mm];
            int scale;
            if (f.cslot[x] >= 0 && f.cslot[y] < 0) scale = f.cslot[x];
            else if (f.cslot[y] >= 0 && f.cslot[x] < 0) scale = f.cslot[y];
            else continue;
            gauge[0] = scale;
            gauge[1] = f.cslot[bb];
            break;
        }
    }
    *nconst = f.nconst;
    return m;
}

}  // namespace

extern "C" {

/* compile_program: returns the word count (HALT included), -1 unsupported,
   -2 stack overflow (peak > 56), -3 `cap` too small, -4 malformed tree.
   `lowered` receives 1 when `lower` rewrote the tree. */
int rch_compile_program(const int *ops, const double *vals, int nn, uint32_t *words, int cap,
                        int *lowered)
{
    Node t;
    if (!load(ops, vals, nn, t)) return -4;
    bool changed = false;
    Node l = lower(t, changed);
    int cur = 0, peak = 0;
    peak_walk(l, cur, peak);
    if (peak > HOST_MAX_STACK) return -2;
    std::vector<uint32_t> out;
    if (!emit(l, out)) return -1;
    out.push_back(HALT);
    if ((int)out.size() > cap) return -3;
    memcpy(words, out.data(), sizeof(uint32_t) * out.size());
    if (lowered) *lowered = changed ? 1 : 0;
    return (int)out.size();
}

/* peak_stack of the lowered tree. */
int rch_peak_stack(const int *ops, const double *vals, int nn)
{
    Node t;
    if (!load(ops, vals, nn, t)) return -4;
    bool changed = false;
    Node l = lower(t, changed);
    int cur = 0, peak = 0;
    peak_walk(l, cur, peak);
    return peak;
}

/* gpu_fit_plan_reason. Writes 4 words per node into `words` (cap words), the
   constants in slot order into c0 (cap_c entries) and the correlation gauge
   (scale, offset; -1 when absent) into gauge[2]. Returns the node count, or a
   negative rejection: -1 too many constants (> 20), -2 too many nodes (> 96),
   -3 no constants, -5 unsupported operator, -6 capacity, -4 malformed tree.
   `allow_no_constants` accepts a constant-free tree (the implicit score and
   gradient entry points take such programs). */
int rch_fit_plan(const int *ops, const double *vals, int nn, uint32_t *words, int cap,
                 double *c0, int cap_c, int *gauge, int *nconst, int allow_no_constants)
{
    Node t;
    if (!load(ops, vals, nn, t)) return -4;
    return plan_tree(t, words, cap, c0, cap_c, gauge, nconst, allow_no_constants);
}

/* rch_fit_plan of a postfix program (`len` words, up to its HALT) instead of
   a pre-order tree: the same plan and the same rejections, -4 for a
   malformed program. */
int rch_fit_plan_postfix(const uint32_t *prog, int len, uint32_t *words, int cap, double *c0,
                         int cap_c, int *gauge, int *nconst, int allow_no_constants)
{
    Node t;
    if (!prog || len <= 0 || !load_postfix(prog, len, t)) return -4;
    return plan_tree(t, words, cap, c0, cap_c, gauge, nconst, allow_no_constants);
}

/* rch_fit_plan_postfix of `nprog` programs, row i of prog[nprog][width]:
   status[i] = its node count or rejection; its plan at words + 4 * width * i
   (4 * width words), c0 + width * i, gauge + 2 * i and nconst[i]. Returns
   the number of accepted programs, or -1 for a bad argument. */
int rch_fit_plans_postfix(int nprog, const uint32_t *prog, int width, uint32_t *words,
                          double *c0, int *gauge, int *nconst, int *status,
                          int allow_no_constants)
{
    if (nprog < 0 || width <= 0 || !prog || !words || !c0 || !gauge || !nconst || !status)
        return -1;
    int ok = 0;
    for (int i = 0; i < nprog; ++i) {
        status[i] = rch_fit_plan_postfix(prog + (size_t)width * i, width,
                                         words + (size_t)4 * width * i, 4 * width,
                                         c0 + (size_t)width * i, width, gauge + 2 * i,
                                         nconst + i, allow_no_constants);
        if (status[i] >= 0) ++ok;
    }
    return ok;
}

/* Writes c[0..k) into the constant operands of a postfix program in place
   (the i-th CONST word's operand becomes the f32 rounding of c[i], the
   order of the tree's pre-order constant slots), which is what compiling the
   tree with those constants emits for a program without inverse
   hyperbolics. Returns the number of constants, -4 for a malformed program,
   -2 when its stack grows past the host limit (the compiler refuses such a
   program), -3 when it holds fewer than k constants; the words change only
   on success, when those after the HALT are reset to HALT (as a caller
   writing the compiled program into a fixed-width slot leaves them). */
int rch_set_postfix_constants(uint32_t *w, int len, const double *c, int k)
{
    if (!w || len <= 0 || k < 0 || (k > 0 && !c)) return -4;
    std::vector<int> at;
    int depth = 0, peak = 0, i = 0;
    for (;;) {
        if (i >= len) return -4;
        const int op = (int)w[i++];
        if (op == HALT) break;
        if (op == CONST || op == VAR) {
            if (i >= len) return -4;
            if (op == CONST) at.push_back(i);
            ++i;
            peak = std::max(peak, ++depth);
            continue;
        }
        const int a = arity(op);
        if (!known(op) || op == ASINH || op == ACOSH || op == ATANH || depth < a) return -4;
        depth -= a - 1;
    }
    if (depth != 1) return -4;
    if (peak > HOST_MAX_STACK) return -2;
    if ((int)at.size() < k) return -3;
    for (int j = 0; j < k; ++j) {
        const float f = (float)c[j];
        memcpy(&w[at[j]], &f, 4);
    }
    for (int j = i; j < len; ++j) w[j] = HALT;
    return (int)at.size();
}

/* rch_set_postfix_constants on rows[r] of words[][width] with c + kmax * r
   and k[r] constants, for r < nrec; status[r] gets each answer. Returns the
   number of rows written. */
int rch_set_postfix_constants_rows(int nrec, uint32_t *words, int width, const int *rows,
                                   const double *c, int kmax, const int *k, int *status)
{
    if (nrec < 0 || width <= 0 || !words || !rows || !c || !k || !status) return -1;
    int done = 0;
    for (int r = 0; r < nrec; ++r) {
        status[r] = rch_set_postfix_constants(words + (size_t)width * rows[r], width,
                                              c + (size_t)kmax * r, k[r]);
        if (status[r] >= 0) ++done;
    }
    return done;
}

/* my-version/src/search.rs:3006-3031 `admission_count`: how many of an
   island's offspring enter the fitted batch. From 2^20 training rows every
   candidate with constants; below, a quarter of the island floored at 32 and
   capped at the island size. */
int rch_admission_count(int island_pop, long long train_rows)
{
    if (island_pop < 1) island_pop = 1;
    if (train_rows >= (1LL << 20)) return island_pop;
    int k = island_pop / 4;
    if (k < 32) k = 32;
    if (k > island_pop) k = island_pop;
    return k < 1 ? 1 : k;
}

/* search.rs:3033-3074 `select_promoted`: per island, the pending offspring
   that have constants, ranked by screened error, then complexity, then
   population index; the best admission_count(island_pop) of each island are
   promoted. The result is (island, index) pairs in ascending order. Errors
   are compared with NaN treated as larger than every number (a total order;
   screening reports +inf, not NaN, for a failed candidate). Returns the count,
   or -1 when `cap` is too small. */
int rch_select_promoted(int nislands, const int *island_pop, int npending, const int *pend_island,
                        const int *pend_index, const double *error, const double *complexity,
                        const unsigned char *has_constants, long long train_rows, int *out_island,
                        int *out_index, int cap)
{
    struct Cand {
        int j;
        double err, cx;
    };
    auto key_lt = [](double a, double b) {
        const bool na = std::isnan(a), nb = std::isnan(b);
        if (na || nb) return !na && nb;
        return a < b;
    };
    std::vector<std::pair<int, int>> out;
    for (int i = 0; i < nislands; ++i) {
        std::vector<Cand> ranked;
        for (int k = 0; k < npending; ++k)
            if (pend_island[k] == i && has_constants[k])
                ranked.push_back({pend_index[k], error[k], complexity[k]});
        std::stable_sort(ranked.begin(), ranked.end(), [&](const Cand &a, const Cand &b) {
            if (key_lt(a.err, b.err)) return true;
            if (key_lt(b.err, a.err)) return false;
            if (key_lt(a.cx, b.cx)) return true;
            if (key_lt(b.cx, a.cx)) return false;
            return a.j < b.j;
        });
        const int take = std::min<int>(rch_admission_count(island_pop[i], train_rows),
                                       (int)ranked.size());
        for (int q = 0; q < take; ++q) out.push_back({i, ranked[q].j});
    }
    std::sort(out.begin(), out.end());
    if ((int)out.size() > cap) return -1;
    for (size_t q = 0; q < out.size(); ++q) {
        out_island[q] = out[q].first;
        out_index[q] = out[q].second;
    }
    return (int)out.size();
}

}  /* extern "C" */
