// CPU restatement of the reference's flat postfix variation engine.
//
// TEST INFRASTRUCTURE ONLY: the checker of the device variation
// (rc_pool_vary). It follows, function by function:
//   my-version/src/genome.rs:43-52    postfix_hash (FNV-1a up to and including HALT)
//   my-version/src/genome.rs:216-302  Philox4x32-10, at(), set_draw(), unit(), below()
//   my-version/src/postfix.rs:84-167  Arena slots, set_slot, key() order, best()
//   my-version/src/postfix.rs:270-313 spans (strict parse)
//   my-version/src/postfix.rs:403-410 front_pick
//   my-version/src/postfix.rs:451-871 Variation: next_generation_with_front,
//                                     fill_random, fill_child, crossover_into,
//                                     mutate_into, edit, random_terminal,
//                                     random_program, gen_subtree
//   my-version/src/postfix.rs:897-957 logical_len, scan_into, splice
//   my-version/src/postfix.rs:962-973 tournament
// Compiled -ffp-contract=off (Rust's f64 semantics).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_set>
#include <vector>

namespace {

const uint32_t HALT = 255, CONST_ = 0, VAR_ = 1;

int opcode_arity(uint32_t w)  // gpu.rs:498-509
{
    switch (w) {
        case 17: case 9: case 10: case 12: case 11: case 6: case 7: case 8: case 21:
        case 22: case 13: case 14: case 19: case 18: case 15: case 16: case 23: case 24:
        case 25: case 33: case 28: case 29: case 42:
            return 1;
        case 2: case 3: case 4: case 5: case 20: case 26: case 27: case 30: case 31:
        case 34: case 35: case 36: case 37: case 38: case 39: case 40: case 41:
            return 2;
        case 32:
            return 3;
        default:
            return -1;
    }
}

uint64_t postfix_hash(const uint32_t *w, size_t n)
{
    uint64_t h = 0xcbf29ce484222325ULL;
    for (size_t i = 0; i < n; ++i) {
        h ^= (uint64_t)w[i];
        h *= 0x00000100000001b3ULL;
        if (w[i] == HALT) break;
    }
    return h;
}

struct Philox {
    uint32_t key[2];
    uint32_t ctr[4];
    static Philox at(uint32_t seed, uint32_t island, uint32_t gen, uint32_t slot)
    {
        Philox p;
        p.key[0] = seed;
        p.key[1] = island;
        p.ctr[0] = gen;
        p.ctr[1] = slot;
        p.ctr[2] = 0;
        p.ctr[3] = 0;
        return p;
    }
    void next(uint32_t out[4])
    {
        uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
        uint32_t k0 = key[0], k1 = key[1];
        for (int r = 0; r < 10; ++r) {
            const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
            const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
            const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
            const uint32_t n1 = (uint32_t)p1;
            const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
            const uint32_t n3 = (uint32_t)p0;
            c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        ctr[3] += 1;
        for (int i = 0; i < 4; ++i) out[i] = c[i];
    }
    uint32_t first()
    {
        uint32_t o[4];
        next(o);
        return o[0];
    }
    double unit() { return (double)first() / 4294967296.0; }
    size_t below(size_t n) { return n == 0 ? 0 : (size_t)first() % n; }
};

struct Span {
    size_t start, end, arity;
};

size_t logical_len(const uint32_t *p, size_t n)
{
    for (size_t i = 0; i < n; ++i)
        if (p[i] == HALT) return i + 1;
    return n;
}

bool spans_strict(const std::vector<uint32_t> &prog, std::vector<Span> &out)
{
    out.clear();
    std::vector<size_t> stack;
    size_t i = 0;
    while (i < prog.size()) {
        const uint32_t w = prog[i];
        if (w == HALT) break;
        if (w == CONST_ || w == VAR_) {
            if (i + 1 >= prog.size() || prog[i + 1] == HALT) return false;
            out.push_back({i, i + 2, 0});
            stack.push_back(i);
            i += 2;
        } else {
            const int a = opcode_arity(w);
            if (a <= 0 || stack.size() < (size_t)a) return false;
            const size_t start = stack[stack.size() - a];
            stack.resize(stack.size() - a);
            out.push_back({start, i + 1, (size_t)a});
            stack.push_back(start);
            i += 1;
        }
    }
    return stack.size() == 1 && i != 0;
}

bool scan_into(const std::vector<uint32_t> &prog, std::vector<Span> &out)
{
    out.clear();
    std::vector<size_t> stack;
    bool saw_halt = false;
    size_t i = 0;
    while (i < prog.size()) {
        const uint32_t w = prog[i];
        if (w == HALT) {
            saw_halt = true;
            break;
        }
        if (w == CONST_ || w == VAR_) {
            if (i + 1 >= prog.size()) return false;
            out.push_back({i, i + 2, 0});
            stack.push_back(i);
            i += 2;
        } else {
            const int a = opcode_arity(w);
            if (a <= 0 || stack.size() < (size_t)a) return false;
            const size_t start = stack[stack.size() - a];
            stack.resize(stack.size() - a);
            out.push_back({start, i + 1, (size_t)a});
            stack.push_back(start);
            i += 1;
        }
    }
    return saw_halt && stack.size() == 1 && !out.empty();
}

bool splice(std::vector<uint32_t> &prog, Span s, const uint32_t *rep, size_t rlen, size_t width)
{
    const size_t old_len = prog.size();
    const size_t new_len = old_len - (s.end - s.start) + rlen;
    if (new_len > width || new_len < 2) return false;
    std::vector<uint32_t> out;
    out.reserve(new_len);
    out.insert(out.end(), prog.begin(), prog.begin() + s.start);
    out.insert(out.end(), rep, rep + rlen);
    out.insert(out.end(), prog.begin() + s.end, prog.end());
    prog.swap(out);
    return true;
}

struct Arena {
    size_t width, islands, pop;
    std::vector<uint32_t> words;
    std::vector<uint16_t> len, cost;
    std::vector<uint64_t> hash;
    std::vector<double> err;
    Arena(size_t w, size_t is, size_t p)
        : width(w), islands(is), pop(p), words(is * p * w, HALT), len(is * p, 0),
          cost(is * p, 0), hash(is * p, 0), err(is * p, NAN)
    {
    }
    size_t idx(size_t i, size_t j) const { return i * pop + j; }
    const uint32_t *slot(size_t k) const { return words.data() + k * width; }
    bool set_slot(size_t k, const std::vector<uint32_t> &prog)
    {
        if (prog.size() < 2 || prog.size() > width) return false;
        std::vector<Span> sp;
        if (!spans_strict(prog, sp)) return false;
        std::fill(words.begin() + k * width, words.begin() + (k + 1) * width, HALT);
        std::copy(prog.begin(), prog.end(), words.begin() + k * width);
        len[k] = (uint16_t)prog.size();
        cost[k] = (uint16_t)std::min<size_t>(sp.size(), 65535);
        hash[k] = postfix_hash(prog.data(), prog.size());
        return true;
    }
    struct Key {
        uint8_t nan;
        uint64_t bits;
        uint16_t cost;
        size_t index;
        bool operator<(const Key &o) const
        {
            if (nan != o.nan) return nan < o.nan;
            if (bits != o.bits) return bits < o.bits;
            if (cost != o.cost) return cost < o.cost;
            return index < o.index;
        }
    };
    Key key(size_t k) const
    {
        const double e = err[k];
        uint64_t bits = 0;
        if (!std::isnan(e)) {
            uint64_t b;
            std::memcpy(&b, &e, 8);
            bits = (b >> 63) ? ~b : (b | (1ULL << 63));
        }
        return {(uint8_t)(std::isnan(e) ? 1 : 0), bits, cost[k], k};
    }
    size_t best(size_t i) const
    {
        size_t b = i * pop;
        for (size_t k = i * pop + 1; k < (i + 1) * pop; ++k)
            if (key(k) < key(b)) b = k;
        return b;
    }
    size_t tournament(size_t i, Philox &rng, size_t k) const
    {
        const size_t base = i * pop;
        size_t best_ = base + rng.below(pop);
        for (size_t t = 1; t < (k < 1 ? 1 : k); ++t) {
            const size_t c = base + rng.below(pop);
            if (key(c) < key(best_)) best_ = c;
        }
        return best_;
    }
};

struct Engine {
    size_t width, nvars, max_complexity, init_depth;
    uint32_t seed;
    bool dedup;
    std::vector<uint32_t> codes;
    std::vector<size_t> by_arity[4];
    std::vector<std::vector<uint32_t>> front;
    double front_p;

    void terminal(Philox &rng, uint32_t t[2]) const
    {
        if (nvars > 0 && rng.unit() < 0.65) {
            t[0] = VAR_;
            t[1] = (uint32_t)rng.below(nvars);
        } else {
            const double v = std::round((rng.unit() * 4.0 - 2.0) * 1000.0) / 1000.0;
            const float f = (float)v;
            std::memcpy(&t[1], &f, 4);
            t[0] = CONST_;
        }
    }
    void gen_subtree(Philox &rng, size_t depth, size_t budget, std::vector<uint32_t> &out) const
    {
        uint32_t t[2];
        if (depth == 0 || budget <= 1 || rng.unit() < 0.15) {
            terminal(rng, t);
            out.push_back(t[0]);
            out.push_back(t[1]);
            return;
        }
        size_t arity;
        if (rng.unit() < 0.35) arity = 1;
        else if (rng.unit() < 0.75) arity = 2;
        else arity = 3;
        const std::vector<size_t> &pool = by_arity[arity];
        if (pool.empty() || budget < arity + 1) {
            terminal(rng, t);
            out.push_back(t[0]);
            out.push_back(t[1]);
            return;
        }
        const uint32_t code = codes[pool[rng.below(pool.size())]];
        const size_t remaining = budget - 1 - arity;
        for (size_t k = 0; k < arity; ++k) {
            const size_t left = arity - k;
            size_t share = remaining / left;
            if (share < 1) share = 1;
            gen_subtree(rng, depth - 1, share, out);
        }
        out.push_back(code);
    }
    std::vector<uint32_t> random_program(Philox &rng, size_t depth) const
    {
        size_t budget = std::min(max_complexity, (width - 1) / 2);
        if (budget < 1) budget = 1;
        std::vector<uint32_t> out;
        gen_subtree(rng, depth, budget, out);
        out.push_back(HALT);
        return out;
    }
    bool front_pick(Philox &rng, size_t &fi) const
    {
        if (front_p > 0.0 && !front.empty() && rng.unit() < front_p) {
            fi = rng.below(front.size());
            return true;
        }
        return false;
    }
    void crossover(std::vector<uint32_t> &prog, const std::vector<uint32_t> &other,
                   Philox &rng) const
    {
        std::vector<Span> a, b;
        if (!scan_into(prog, a)) return;
        if (!scan_into(other, b)) return;
        if (a.empty() || b.empty()) return;
        const size_t ai = rng.below(a.size());
        const size_t bi = rng.below(b.size());
        const Span sa = a[ai], sb = b[bi];
        std::vector<uint32_t> rep(other.begin() + sb.start, other.begin() + sb.end);
        splice(prog, sa, rep.data(), rep.size(), width);
    }
    bool edit(std::vector<uint32_t> &prog, const std::vector<Span> &sp, int kind,
              Philox &rng) const
    {
        auto eligible = [&](const Span &s) {
            return kind == 0 ? s.arity > 0 : (kind == 1 ? s.arity == 0 : true);
        };
        size_t count = 0;
        for (const Span &s : sp)
            if (eligible(s)) ++count;
        if (count == 0) return false;
        size_t target = rng.below(count), node = 0;
        for (size_t i = 0, seen = 0; i < sp.size(); ++i) {
            if (!eligible(sp[i])) continue;
            if (seen == target) {
                node = i;
                break;
            }
            ++seen;
        }
        const Span s = sp[node];
        if (kind == 0) {
            const std::vector<size_t> &pool = by_arity[s.arity < 3 ? s.arity : 3];
            if (pool.size() < 2) return false;
            const uint32_t current = prog[s.end - 1];
            size_t n = 0;
            for (size_t k : pool)
                if (codes[k] != current) ++n;
            if (n == 0) return false;
            const size_t want = rng.below(n);
            uint32_t pick = 0;
            size_t m = 0;
            for (size_t k : pool) {
                if (codes[k] == current) continue;
                if (m == want) {
                    pick = codes[k];
                    break;
                }
                ++m;
            }
            prog[s.end - 1] = pick;
            return true;
        }
        if (kind == 1) {
            uint32_t t[2];
            terminal(rng, t);
            prog[s.start] = t[0];
            prog[s.start + 1] = t[1];
            return true;
        }
        const size_t budget = (width > 0 ? width - 1 : 0) - (prog.size() - s.end);
        if (budget < 2) return false;
        std::vector<uint32_t> tmp;
        gen_subtree(rng, init_depth, budget, tmp);
        if (s.end - s.start + tmp.size() > width) return false;
        return splice(prog, s, tmp.data(), tmp.size(), width);
    }
    void mutate(std::vector<uint32_t> &prog, Philox &rng) const
    {
        std::vector<Span> sp;
        if (!scan_into(prog, sp) || sp.empty()) return;
        const double r = rng.unit();
        int order[3];
        if (r < 0.25) { order[0] = 0; order[1] = 2; order[2] = 1; }
        else if (r < 0.6) { order[0] = 1; order[1] = 0; order[2] = 2; }
        else { order[0] = 2; order[1] = 0; order[2] = 1; }
        for (int kind : order)
            if (edit(prog, sp, kind, rng)) return;
    }
    void fill_random(Arena &next, size_t i, size_t j, uint32_t gen, uint64_t salt) const
    {
        Philox rng = Philox::at(seed, (uint32_t)i, gen, (uint32_t)j);
        uint32_t o[4];
        for (uint64_t s = 0; s < salt; ++s) rng.next(o);
        std::vector<uint32_t> best;
        bool have = false;
        for (int t = 0; t < 8; ++t) {
            std::vector<uint32_t> prog = random_program(rng, init_depth);
            std::vector<Span> sp;
            if (spans_strict(prog, sp)) {
                if (sp.size() <= max_complexity && prog.size() <= width) {
                    best = prog;
                    have = true;
                    break;
                }
            }
        }
        if (!have) best = {VAR_, 0, HALT};
        const size_t k = next.idx(i, j);
        next.set_slot(k, best);
        next.err[k] = NAN;
    }
    std::vector<uint32_t> slot_program(const Arena &a, size_t k) const
    {
        const uint32_t *s = a.slot(k);
        return std::vector<uint32_t>(s, s + logical_len(s, a.width));
    }
    void fill_child(Arena &next, const Arena &parents, std::unordered_set<uint64_t> &seen,
                    size_t i, size_t j, uint32_t gen) const
    {
        for (uint32_t attempt = 0; attempt < 64; ++attempt) {
            Philox rng = Philox::at(seed, (uint32_t)i, gen, (uint32_t)j);
            if (attempt > 0) rng.ctr[2] = attempt;
            std::vector<uint32_t> prog;
            size_t fi;
            if (front_pick(rng, fi)) {
                const std::vector<uint32_t> &f = front[fi];
                prog.assign(f.begin(), f.begin() + logical_len(f.data(), f.size()));
            } else {
                prog = slot_program(parents, parents.tournament(i, rng, 4));
            }
            if (rng.unit() < 0.5) {
                if (front_pick(rng, fi)) {
                    const std::vector<uint32_t> &f = front[fi];
                    std::vector<uint32_t> other(f.begin(),
                                                f.begin() + logical_len(f.data(), f.size()));
                    crossover(prog, other, rng);
                } else {
                    const size_t o = parents.tournament(i, rng, 4);
                    crossover(prog, slot_program(parents, o), rng);
                }
            }
            mutate(prog, rng);
            if (rng.unit() < 0.5) mutate(prog, rng);
            std::vector<Span> sp;
            if (prog.size() > width || !scan_into(prog, sp)) continue;
            if (sp.size() > max_complexity) continue;
            const uint64_t h = postfix_hash(prog.data(), prog.size());
            if (dedup && !seen.insert(h).second) continue;
            if (next.set_slot(next.idx(i, j), prog)) return;
        }
        fill_random(next, i, j, gen, 64);
    }
};

}  // namespace

extern "C" {

/* The first `n` Philox outputs at (seed, island, gen, slot) with draw index
   `draw` (counter word 2): out[4n]. */
void orv_philox(uint32_t seed, uint32_t island, uint32_t gen, uint32_t slot, uint32_t draw,
                int n, uint32_t *out)
{
    Philox p = Philox::at(seed, island, gen, slot);
    p.ctr[2] = draw;
    for (int i = 0; i < n; ++i) p.next(out + 4 * i);
}

uint64_t orv_hash(const uint32_t *w, int n) { return postfix_hash(w, (size_t)n); }

/* Number of nodes of the strict parse, or -1 (postfix.rs:270-313). */
int orv_spans(const uint32_t *w, int n)
{
    std::vector<uint32_t> p(w, w + n);
    std::vector<Span> s;
    return spans_strict(p, s) ? (int)s.size() : -1;
}

static Engine make_engine(int width, int nvars, int max_complexity, uint32_t seed, int init_depth,
                          int dedup, const uint32_t *ops, int nops, const uint32_t *front,
                          const uint32_t *front_off, int nfront, double front_p)
{
    Engine e;
    e.width = (size_t)width;
    e.nvars = (size_t)nvars;
    e.max_complexity = (size_t)max_complexity;
    e.seed = seed;
    e.init_depth = (size_t)init_depth;
    e.dedup = dedup != 0;
    for (int k = 0; k < nops; ++k) {
        e.codes.push_back(ops[2 * k]);
        e.by_arity[ops[2 * k + 1] & 3].push_back((size_t)k);
    }
    for (int f = 0; f < nfront; ++f)
        e.front.emplace_back(front + front_off[f], front + front_off[f + 1]);
    e.front_p = front_p;
    return e;
}

/* A parent arena as the reference's tests build one: consecutive random
   programs from one generator at (seed, 0, 0, 0), a malformed one redrawn.
   out[count * width], HALT padded. */
void orv_random_arena(int width, int nvars, int max_complexity, uint32_t seed, int init_depth,
                      const uint32_t *ops, int nops, uint32_t rng_seed, int depth, int count,
                      uint32_t *out)
{
    Engine e = make_engine(width, nvars, max_complexity, seed, init_depth, 1, ops, nops, nullptr,
                           nullptr, 0, 0.0);
    Philox rng = Philox::at(rng_seed, 0, 0, 0);
    Arena a((size_t)width, 1, (size_t)count);
    for (int i = 0; i < count; ++i) {
        std::vector<uint32_t> p = e.random_program(rng, (size_t)depth);
        std::vector<Span> s;
        while (!spans_strict(p, s)) p = e.random_program(rng, (size_t)depth);
        a.set_slot((size_t)i, p);
    }
    std::memcpy(out, a.words.data(), sizeof(uint32_t) * a.words.size());
}

/* Variation::next_generation_with_front (postfix.rs:519-567) of a parent
   arena given as HALT-padded slots and errors. Outputs the child arena. */
int orv_next_generation(int width, int nvars, int max_complexity, uint32_t seed, int init_depth,
                        int dedup, const uint32_t *ops, int nops, int islands, int pop,
                        const uint32_t *words, const double *err, uint32_t gen,
                        const uint8_t *restart, const uint32_t *front, const uint32_t *front_off,
                        int nfront, double front_p, uint32_t *out_words, uint16_t *out_len,
                        uint16_t *out_cost, uint64_t *out_hash, double *out_err)
{
    Engine e = make_engine(width, nvars, max_complexity, seed, init_depth, dedup, ops, nops, front,
                           front_off, nfront, front_p);
    Arena parents((size_t)width, (size_t)islands, (size_t)pop);
    for (size_t k = 0; k < (size_t)islands * pop; ++k) {
        const uint32_t *s = words + k * width;
        std::vector<uint32_t> p(s, s + logical_len(s, (size_t)width));
        if (!parents.set_slot(k, p)) return -1;
        parents.err[k] = err[k];
    }
    Arena next((size_t)width, (size_t)islands, (size_t)pop);
    std::unordered_set<uint64_t> seen;
    for (size_t k = 0; k < parents.hash.size(); ++k) seen.insert(parents.hash[k]);
    for (size_t i = 0; i < (size_t)islands; ++i) {
        if (restart && restart[i]) {
            for (size_t j = 0; j < (size_t)pop; ++j) e.fill_random(next, i, j, gen, 0);
            continue;
        }
        const size_t elite = parents.best(i), d = next.idx(i, 0);
        std::copy(parents.words.begin() + elite * width, parents.words.begin() + (elite + 1) * width,
                  next.words.begin() + d * width);
        next.len[d] = parents.len[elite];
        next.cost[d] = parents.cost[elite];
        next.hash[d] = parents.hash[elite];
        next.err[d] = parents.err[elite];
        for (size_t j = 1; j < (size_t)pop; ++j) e.fill_child(next, parents, seen, i, j, gen);
    }
    std::memcpy(out_words, next.words.data(), sizeof(uint32_t) * next.words.size());
    std::memcpy(out_len, next.len.data(), sizeof(uint16_t) * next.len.size());
    std::memcpy(out_cost, next.cost.data(), sizeof(uint16_t) * next.cost.size());
    std::memcpy(out_hash, next.hash.data(), sizeof(uint64_t) * next.hash.size());
    std::memcpy(out_err, next.err.data(), sizeof(double) * next.err.size());
    return 0;
}

}  // extern "C"
