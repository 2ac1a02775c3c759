/*
 * The flat postfix variation engine, compiled for the device and the host.
 *
 * One child of the next generation is a pure function of its position
 * (seed, island, generation, slot, attempt): every random decision comes from
 * a Philox4x32-10 counter stream at that position (genome.rs:216-302), the
 * parents are read from the fixed-width pool, and the program is built in a
 * per-thread buffer. The same code runs on the device for the bulk of a
 * generation (every slot's first attempts in parallel) and on the host for
 * the rare later attempts the order-dependent duplicate rule asks for, so the
 * two agree bit for bit. Operations follow the reference engine
 * (postfix.rs:451-871, :897-973): tournament by (error, cost, slot), one
 * optional crossover, one or two mutations (operator change, terminal
 * resample, subtree replacement), and the validity, size and complexity
 * checks. Only integer arithmetic and exactly rounded f64 operations are
 * used (no contraction), so host and device results are identical.
 */
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#ifndef __CUDACC__
#define __host__
#define __device__
#endif

#define RV_WMAX 128    /* widest slot the engine handles (words) */
#define RV_MAXOPS 64   /* operator table entries */
#define RV_HALT 255u
#define RV_CONST 0u
#define RV_VAR 1u

/* The engine's configuration (Variation::new, postfix.rs:454-498). */
struct RvConfig {
    int width, nvars, max_complexity, init_depth, dedup;
    unsigned int seed, gen;
    int islands, pop;
    int nops;
    unsigned int code[RV_MAXOPS];
    int by_arity[4][RV_MAXOPS]; /* table indexes per arity */
    int n_arity[4];
    int nfront;
    double front_p;
};

/* ---- Philox4x32-10 at a position --------------------------------------- */

struct RvPhilox {
    uint32_t key0, key1;
    uint32_t c0, c1, c2, c3;
};

__host__ __device__ inline uint32_t rv_mulhi(uint32_t a, uint32_t b)
{
    return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
}

__host__ __device__ inline RvPhilox rv_at(uint32_t seed, uint32_t island, uint32_t gen,
                                          uint32_t slot)
{
    RvPhilox p;
    p.key0 = seed;
    p.key1 = island;
    p.c0 = gen;
    p.c1 = slot;
    p.c2 = 0;
    p.c3 = 0;
    return p;
}

/* The first word of the next block; the counter's last word advances. */
__host__ __device__ inline uint32_t rv_next(RvPhilox &p)
{
    uint32_t c0 = p.c0, c1 = p.c1, c2 = p.c2, c3 = p.c3;
    uint32_t k0 = p.key0, k1 = p.key1;
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = rv_mulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = rv_mulhi(0xCD9E8D57u, c2);
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    p.c3 += 1;
    return c0;
}

__host__ __device__ inline double rv_unit(RvPhilox &p) { return (double)rv_next(p) / 4294967296.0; }

__host__ __device__ inline int rv_below(RvPhilox &p, int n)
{
    return n <= 0 ? 0 : (int)(rv_next(p) % (uint32_t)n);
}

/* ---- parsing --------------------------------------------------------------- */

__host__ __device__ inline int rv_arity(uint32_t w)
{
    if (w == 32u) return 3;
    if ((w >= 2u && w <= 5u) || w == 20u || w == 26u || w == 27u || w == 30u || w == 31u ||
        (w >= 34u && w <= 41u))
        return 2;
    if ((w >= 6u && w <= 19u) || w == 21u || w == 22u || w == 23u || w == 24u || w == 25u ||
        w == 28u || w == 29u || w == 33u || w == 42u)
        return 1;
    return -1;
}

/* A node of a parsed program: its word span and arity (start | end << 8 |
   arity << 16; every index is below RV_WMAX). */
__host__ __device__ inline int rv_start(uint32_t s) { return (int)(s & 0xffu); }
__host__ __device__ inline int rv_end(uint32_t s) { return (int)((s >> 8) & 0xffu); }
__host__ __device__ inline int rv_sarity(uint32_t s) { return (int)(s >> 16); }

/* Parse `prog[0..n)` into its nodes (postfix.rs:904-944 scan_into when
   `strict` is false: a HALT is required; postfix.rs:270-313 spans when
   `strict`: a terminal's operand may not be HALT and a HALT is optional).
   Returns the node count, or -1 when malformed. */
__host__ __device__ inline int rv_parse(const uint32_t *prog, int n, uint32_t *spans, bool strict)
{
    uint8_t stack[RV_WMAX];
    int sp = 0, ns = 0, i = 0;
    bool saw_halt = false;
    while (i < n) {
        const uint32_t w = prog[i];
        if (w == RV_HALT) {
            saw_halt = true;
            break;
        }
        if (w == RV_CONST || w == RV_VAR) {
            if (i + 1 >= n) return -1;
            if (strict && prog[i + 1] == RV_HALT) return -1;
            spans[ns++] = (uint32_t)i | ((uint32_t)(i + 2) << 8);
            stack[sp++] = (uint8_t)i;
            i += 2;
        } else {
            const int a = rv_arity(w);
            if (a <= 0 || sp < a) return -1;
            const int start = stack[sp - a];
            sp -= a;
            spans[ns++] = (uint32_t)start | ((uint32_t)(i + 1) << 8) | ((uint32_t)a << 16);
            stack[sp++] = (uint8_t)start;
            i += 1;
        }
    }
    if (strict) return (sp == 1 && i != 0) ? ns : -1;
    return (saw_halt && sp == 1 && ns > 0) ? ns : -1;
}

__host__ __device__ inline int rv_logical_len(const uint32_t *p, int n)
{
    for (int i = 0; i < n; ++i)
        if (p[i] == RV_HALT) return i + 1;
    return n;
}

__host__ __device__ inline uint64_t rv_hash(const uint32_t *w, int n)
{
    uint64_t h = 0xcbf29ce484222325ULL;
    for (int i = 0; i < n; ++i) {
        h ^= (uint64_t)w[i];
        h *= 0x00000100000001b3ULL;
        if (w[i] == RV_HALT) break;
    }
    return h;
}

/* Replace node `s` of prog (length *n) by rep[0..rn) (postfix.rs:946-957). */
__host__ __device__ inline bool rv_splice(uint32_t *prog, int *n, uint32_t s, const uint32_t *rep,
                                          int rn, int width)
{
    const int a = rv_start(s), b = rv_end(s);
    const int old_len = *n, new_len = old_len - (b - a) + rn;
    if (new_len > width || new_len < 2) return false;
    if (rn > b - a) {
        for (int k = old_len - 1; k >= b; --k) prog[k + rn - (b - a)] = prog[k];
    } else if (rn < b - a) {
        for (int k = b; k < old_len; ++k) prog[k + rn - (b - a)] = prog[k];
    }
    for (int k = 0; k < rn; ++k) prog[a + k] = rep[k];
    *n = new_len;
    return true;
}

/* ---- parents --------------------------------------------------------------- */

/* The canonical (error, cost, slot) key (postfix.rs:155-167): NaN last, then
   the IEEE total order of the error. */
struct RvKey {
    uint32_t nan;
    uint64_t bits;
    uint32_t cost;
    uint32_t index;
};

__host__ __device__ inline RvKey rv_key(const double *err, const uint16_t *cost, int k)
{
    const double e = err[k];
    RvKey r;
    r.nan = e != e ? 1u : 0u;
    uint64_t b;
    memcpy(&b, &e, 8);
    r.bits = r.nan ? 0ULL : ((b >> 63) ? ~b : (b | (1ULL << 63)));
    r.cost = cost[k];
    r.index = (uint32_t)k;
    return r;
}

__host__ __device__ inline bool rv_less(const RvKey &a, const RvKey &b)
{
    if (a.nan != b.nan) return a.nan < b.nan;
    if (a.bits != b.bits) return a.bits < b.bits;
    if (a.cost != b.cost) return a.cost < b.cost;
    return a.index < b.index;
}

/* Tournament of k = 4 draws within island i (postfix.rs:962-973). */
__host__ __device__ inline int rv_tournament(const RvConfig &c, const double *err,
                                             const uint16_t *cost, int island, RvPhilox &rng)
{
    const int base = island * c.pop;
    int best = base + rv_below(rng, c.pop);
    RvKey kb = rv_key(err, cost, best);
    for (int t = 1; t < 4; ++t) {
        const int k = base + rv_below(rng, c.pop);
        const RvKey kk = rv_key(err, cost, k);
        if (rv_less(kk, kb)) {
            best = k;
            kb = kk;
        }
    }
    return best;
}

/* ---- generation ------------------------------------------------------------ */

/* A terminal (postfix.rs:814-821): an input with probability 0.65 when there
   are inputs, else a constant round((4u - 2) * 1000) / 1000 as f32. */
__host__ __device__ inline void rv_terminal(const RvConfig &c, RvPhilox &rng, uint32_t t[2])
{
    if (c.nvars > 0 && rv_unit(rng) < 0.65) {
        t[0] = RV_VAR;
        t[1] = (uint32_t)rv_below(rng, c.nvars);
        return;
    }
#ifdef __CUDA_ARCH__
    const double v = __ddiv_rn(round(__dmul_rn(__dsub_rn(__dmul_rn(rv_unit(rng), 4.0), 2.0), 1000.0)),
                               1000.0);
    const float f = __double2float_rn(v);
#else
    volatile double u4 = rv_unit(rng) * 4.0;
    volatile double s = u4 - 2.0;
    volatile double m = s * 1000.0;
    const double v = std::round(m) / 1000.0;
    const float f = (float)v;
#endif
    uint32_t bits;
    memcpy(&bits, &f, 4);
    t[0] = RV_CONST;
    t[1] = bits;
}

/* Append a postfix subtree for `budget` nodes and `depth` levels
   (postfix.rs:834-871), written without recursion: a frame per pending
   operator holds its code, arity, the children still to generate and the
   share left for them. As in the reference the children's shares are not
   charged against each other, so a subtree can outgrow its budget; it is
   always generated to the end (the draws it consumes decide what follows),
   words past `cap` are counted in *n but not stored, and the caller rejects
   a result longer than the slot as the reference does. Depth <= 15. */
__host__ __device__ inline void rv_subtree(const RvConfig &c, RvPhilox &rng, int depth, int budget,
                                           uint32_t *out, int *n, int cap)
{
    struct Frame {
        uint32_t code;
        int arity, k, remaining, depth;
    };
    Frame fr[16];
    int top = 0;
    int d = depth, b = budget;
    for (;;) {
        /* generate the node (d, b): a terminal, or push an operator frame */
        bool terminal = d == 0 || b <= 1 || rv_unit(rng) < 0.15;
        int arity = 0;
        if (!terminal) {
            if (rv_unit(rng) < 0.35) arity = 1;
            else if (rv_unit(rng) < 0.75) arity = 2;
            else arity = 3;
            if (c.n_arity[arity] == 0 || b < arity + 1) terminal = true;
        }
        if (terminal) {
            uint32_t t[2];
            rv_terminal(c, rng, t);
            if (*n < cap) out[*n] = t[0];
            if (*n + 1 < cap) out[*n + 1] = t[1];
            *n += 2;
        } else {
            Frame f;
            f.code = c.code[c.by_arity[arity][rv_below(rng, c.n_arity[arity])]];
            f.arity = arity;
            f.k = 0;
            f.remaining = b - 1 - arity;
            f.depth = d - 1;
            fr[top++] = f;
        }
        /* the next child of the innermost open operator, closing finished ones */
        for (;;) {
            if (top == 0) return;
            Frame &f = fr[top - 1];
            if (f.k < f.arity) {
                const int left = f.arity - f.k;
                int share = f.remaining / left;
                if (share < 1) share = 1;
                f.k++;
                d = f.depth;
                b = share;
                break;
            }
            if (*n < cap) out[*n] = f.code;
            ++*n;
            --top;
        }
    }
}

/* random_program (postfix.rs:823-832) into out[0..cap); *n is the full
   length, which may exceed cap. */
__host__ __device__ inline void rv_random_program(const RvConfig &c, RvPhilox &rng, int depth,
                                                  uint32_t *out, int *n, int cap)
{
    int budget = c.max_complexity < (c.width - 1) / 2 ? c.max_complexity : (c.width - 1) / 2;
    if (budget < 1) budget = 1;
    *n = 0;
    rv_subtree(c, rng, depth, budget, out, n, cap);
    if (*n < cap) out[*n] = RV_HALT;
    ++*n;
}

/* One edit of kind 0 (operator), 1 (terminal) or 2 (subtree)
   (postfix.rs:741-812). */
__host__ __device__ inline bool rv_edit(const RvConfig &c, uint32_t *prog, int *n,
                                        const uint32_t *spans, int ns, int kind, RvPhilox &rng,
                                        uint32_t *tmp)
{
    int count = 0;
    for (int i = 0; i < ns; ++i) {
        const int a = rv_sarity(spans[i]);
        if (kind == 0 ? a > 0 : (kind == 1 ? a == 0 : true)) ++count;
    }
    if (count == 0) return false;
    const int target = rv_below(rng, count);
    int node = 0;
    for (int i = 0, seen = 0; i < ns; ++i) {
        const int a = rv_sarity(spans[i]);
        if (!(kind == 0 ? a > 0 : (kind == 1 ? a == 0 : true))) continue;
        if (seen == target) {
            node = i;
            break;
        }
        ++seen;
    }
    const uint32_t s = spans[node];
    if (kind == 0) {
        const int a = rv_sarity(s) < 3 ? rv_sarity(s) : 3;
        if (c.n_arity[a] < 2) return false;
        const uint32_t current = prog[rv_end(s) - 1];
        int m = 0;
        for (int k = 0; k < c.n_arity[a]; ++k)
            if (c.code[c.by_arity[a][k]] != current) ++m;
        if (m == 0) return false;
        const int want = rv_below(rng, m);
        uint32_t pick = 0;
        for (int k = 0, q = 0; k < c.n_arity[a]; ++k) {
            const uint32_t code = c.code[c.by_arity[a][k]];
            if (code == current) continue;
            if (q == want) {
                pick = code;
                break;
            }
            ++q;
        }
        prog[rv_end(s) - 1] = pick;
        return true;
    }
    if (kind == 1) {
        uint32_t t[2];
        rv_terminal(c, rng, t);
        prog[rv_start(s)] = t[0];
        prog[rv_start(s) + 1] = t[1];
        return true;
    }
    const int budget = (c.width > 0 ? c.width - 1 : 0) - (*n - rv_end(s));
    if (budget < 2) return false;
    int tn = 0;
    rv_subtree(c, rng, c.init_depth, budget, tmp, &tn, RV_WMAX);
    if (rv_end(s) - rv_start(s) + tn > c.width) return false;
    return rv_splice(prog, n, s, tmp, tn, c.width);
}

__host__ __device__ inline void rv_mutate(const RvConfig &c, uint32_t *prog, int *n,
                                          uint32_t *spans, RvPhilox &rng, uint32_t *tmp)
{
    const int ns = rv_parse(prog, *n, spans, false);
    if (ns <= 0) return;
    const double r = rv_unit(rng);
    int order[3];
    if (r < 0.25) { order[0] = 0; order[1] = 2; order[2] = 1; }
    else if (r < 0.6) { order[0] = 1; order[1] = 0; order[2] = 2; }
    else { order[0] = 2; order[1] = 0; order[2] = 1; }
    for (int q = 0; q < 3; ++q)
        if (rv_edit(c, prog, n, spans, ns, order[q], rng, tmp)) return;
}

/* front_pick (postfix.rs:403-410). */
__host__ __device__ inline int rv_front_pick(const RvConfig &c, RvPhilox &rng)
{
    if (c.front_p > 0.0 && c.nfront > 0 && rv_unit(rng) < c.front_p) return rv_below(rng, c.nfront);
    return -1;
}

/* Where the parents live: the pool slots with their errors and costs, and
   the front programs. */
struct RvParents {
    const uint32_t *words;
    const double *err;
    const uint16_t *cost;
    const uint32_t *front;
    const uint32_t *front_off;
};

/* Outcome of one attempt. */
enum { RV_REJECT = 0, RV_CANDIDATE = 1, RV_CANDIDATE_NOSLOT = 2 };

/* One attempt of fill_child (postfix.rs:600-667) up to the duplicate test:
   the child program in prog[0..*n), and whether it is rejected before
   hashing, a candidate whose set_slot succeeds, or a candidate whose
   set_slot fails (its hash still enters the duplicate set). */
__host__ __device__ inline int rv_attempt(const RvConfig &c, const RvParents &par, int island,
                                          int slot, int attempt, uint32_t *prog, int *n,
                                          uint32_t *spans, uint32_t *other, uint32_t *tmp,
                                          int *cost_out, uint64_t *hash_out)
{
    RvPhilox rng = rv_at(c.seed, (uint32_t)island, c.gen, (uint32_t)slot);
    if (attempt > 0) rng.c2 = (uint32_t)attempt;
    int fi = rv_front_pick(c, rng);
    if (fi >= 0) {
        const uint32_t *f = par.front + par.front_off[fi];
        const int fl = (int)(par.front_off[fi + 1] - par.front_off[fi]);
        *n = rv_logical_len(f, fl);
        for (int k = 0; k < *n; ++k) prog[k] = f[k];
    } else {
        const int src = rv_tournament(c, par.err, par.cost, island, rng);
        const uint32_t *s = par.words + (size_t)src * c.width;
        *n = rv_logical_len(s, c.width);
        for (int k = 0; k < *n; ++k) prog[k] = s[k];
    }
    if (rv_unit(rng) < 0.5) {
        const uint32_t *o;
        int on;
        fi = rv_front_pick(c, rng);
        if (fi >= 0) {
            o = par.front + par.front_off[fi];
            on = rv_logical_len(o, (int)(par.front_off[fi + 1] - par.front_off[fi]));
        } else {
            const int src = rv_tournament(c, par.err, par.cost, island, rng);
            o = par.words + (size_t)src * c.width;
            on = rv_logical_len(o, c.width);
        }
        /* crossover_into (postfix.rs:680-710) */
        const int na = rv_parse(prog, *n, spans, false);
        if (na >= 0) {
            const int nb = rv_parse(o, on, other, false);
            if (nb >= 0 && na > 0 && nb > 0) {
                const int ai = rv_below(rng, na);
                const int bi = rv_below(rng, nb);
                const uint32_t sa = spans[ai], sb = other[bi];
                for (int k = rv_start(sb); k < rv_end(sb); ++k) tmp[k - rv_start(sb)] = o[k];
                rv_splice(prog, n, sa, tmp, rv_end(sb) - rv_start(sb), c.width);
            }
        }
    }
    rv_mutate(c, prog, n, spans, rng, tmp);
    if (rv_unit(rng) < 0.5) rv_mutate(c, prog, n, spans, rng, tmp);
    if (*n > c.width) return RV_REJECT;
    const int ns = rv_parse(prog, *n, spans, false);
    if (ns < 0 || ns > c.max_complexity) return RV_REJECT;
    *hash_out = rv_hash(prog, *n);
    /* set_slot (postfix.rs:95-110) */
    if (*n < 2) return RV_CANDIDATE_NOSLOT;
    const int strict = rv_parse(prog, *n, spans, true);
    if (strict < 0) return RV_CANDIDATE_NOSLOT;
    *cost_out = strict;
    return RV_CANDIDATE;
}

/* fill_random (postfix.rs:572-597): the first of eight random programs that
   parses, fits and respects the complexity bound, else x0. */
__host__ __device__ inline void rv_random_slot(const RvConfig &c, int island, int slot,
                                               uint32_t salt, uint32_t *prog, int *n,
                                               uint32_t *spans, int *cost_out, uint64_t *hash_out)
{
    RvPhilox rng = rv_at(c.seed, (uint32_t)island, c.gen, (uint32_t)slot);
    for (uint32_t s = 0; s < salt; ++s) rv_next(rng);
    for (int t = 0; t < 8; ++t) {
        int pn = 0;
        rv_random_program(c, rng, c.init_depth, prog, &pn, RV_WMAX);
        if (pn > c.width) continue;
        const int ns = rv_parse(prog, pn, spans, true);
        if (ns >= 0 && ns <= c.max_complexity) {
            *n = pn;
            *cost_out = ns;
            *hash_out = rv_hash(prog, pn);
            return;
        }
    }
    prog[0] = RV_VAR;
    prog[1] = 0;
    prog[2] = RV_HALT;
    *n = 3;
    *cost_out = 1;
    *hash_out = rv_hash(prog, 3);
}
