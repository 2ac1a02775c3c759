/*
 * The next generation of the fixed-width postfix pool, built on the device
 * (my-version/src/postfix.rs:511-567 Variation::next_generation_with_front;
 * the reference runs it on the host and names the CUDA port as its next step).
 *
 * 1. rv_parents: per parent slot its length, node count (the tournament's
 *    tie-break) and FNV-1a hash (genome.rs:43-52).
 * 2. rv_children: every child slot's first RV_K attempts in parallel, one
 *    thread per (slot, attempt): the attempt's program, its outcome (rejected
 *    before hashing / a candidate / a candidate that set_slot refuses), hash,
 *    length and node count. Slots of restarting islands get their random
 *    program instead.
 * 3. The duplicate rule, on the host over these compact arrays: in slot order
 *    each child takes its first attempt whose hash is not yet taken by a
 *    parent or an earlier child (postfix.rs:655-666); this order dependence is
 *    the one sequential step. An attempt beyond the first RV_K, or the random
 *    fallback after 64 attempts, is computed on the host by the same engine
 *    code (vary_gen.cuh), bit for bit what the device would produce.
 * 4. rv_gather: each child slot copies its chosen program (or its island's
 *    elite) into the other pool, HALT padded, with its metadata.
 * Programs never cross PCIe; the host sees hashes and outcomes only, plus
 * the few programs it computed itself.
 */
#include <algorithm>
#include <cstring>
#include <vector>

#include "rc_internal.h"
#include "vary_gen.cuh"

#define RV_K 3   /* attempts per slot computed on the device */
#define RV_T 128

namespace {

/* Parent metadata: logical length, strict node count (-1 when the slot is
   not a valid program), hash. */
__global__ void __launch_bounds__(RV_T) rv_parents(const uint32_t *__restrict__ words, int width,
                                                   int nslots, uint16_t *len, int *cost,
                                                   uint16_t *cost16, unsigned long long *hash,
                                                   int *bad)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nslots) return;
    const uint32_t *s = words + (size_t)k * width;
    uint32_t spans[RV_WMAX];
    const int n = rv_logical_len(s, width);
    const int cst = n >= 2 ? rv_parse(s, n, spans, true) : -1;
    len[k] = (uint16_t)n;
    cost[k] = cst;
    /* the tournament's tie-break key; a slot that is not a valid program
       fails the whole call (the children are not built from it) */
    cost16[k] = (uint16_t)(cst < 0 ? 0 : min(cst, 65535));
    if (cst < 0) atomicOr(bad, 1);
    hash[k] = rv_hash(s, n);
}

/* Outcome of one (slot, attempt) item. */
struct RvItem {
    unsigned long long hash;
    uint16_t len, cost;
    uint8_t status, pad[3];
};

__global__ void __launch_bounds__(RV_T) rv_children(RvConfig c, RvParents par,
                                                    const uint8_t *__restrict__ restart,
                                                    const int *__restrict__ bad, RvItem *items,
                                                    uint32_t *progs)
{
    const int nslots = c.islands * c.pop;
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= nslots * RV_K) return;
    if (*bad) return; /* an invalid parent: the call fails, nothing is built */
    const int k = it / RV_K, attempt = it % RV_K;
    const int island = k / c.pop, slot = k % c.pop;
    uint32_t prog[RV_WMAX], spans[RV_WMAX], other[RV_WMAX], tmp[RV_WMAX];
    RvItem r;
    r.hash = 0;
    r.len = 0;
    r.cost = 0;
    r.status = RV_REJECT;
    int n = 0, cost = 0;
    uint64_t h = 0;
    bool have = false;
    if (restart && restart[island]) {
        if (attempt == 0) {
            rv_random_slot(c, island, slot, 0, prog, &n, spans, &cost, &h);
            r.status = RV_CANDIDATE;
            have = true;
        }
    } else if (slot > 0) {
        r.status = (uint8_t)rv_attempt(c, par, island, slot, attempt, prog, &n, spans, other, tmp,
                                       &cost, &h);
        have = r.status != RV_REJECT;
    }
    if (have) {
        r.hash = h;
        r.len = (uint16_t)n;
        r.cost = (uint16_t)cost;
        uint32_t *dst = progs + (size_t)it * c.width;
        for (int q = 0; q < c.width; ++q) dst[q] = q < n ? prog[q] : RV_HALT;
    }
    items[it] = r;
}

/* Where a child slot's program comes from. */
enum { RV_SRC_ITEM = 0, RV_SRC_HOST = 1, RV_SRC_PARENT = 2 };

struct RvChoice {
    int src, index; /* item index, host program index, or parent slot */
    uint16_t len, cost;
    unsigned long long hash;
    double err;
};

__global__ void __launch_bounds__(RV_T) rv_gather(int width, int nslots,
                                                  const RvChoice *__restrict__ choice,
                                                  const uint32_t *__restrict__ progs,
                                                  const uint32_t *__restrict__ host_progs,
                                                  const uint32_t *__restrict__ parents,
                                                  uint32_t *__restrict__ next)
{
    const size_t total = (size_t)nslots * width;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(q / width), w = (int)(q % width);
        const RvChoice ch = choice[k];
        const uint32_t *src = ch.src == RV_SRC_ITEM ? progs + (size_t)ch.index * width
                              : ch.src == RV_SRC_HOST ? host_progs + (size_t)ch.index * width
                                                      : parents + (size_t)ch.index * width;
        next[q] = src[w];
    }
}

/* Open-addressing set of 64-bit hashes (the reference's HashSet<u64>). */
struct HashSet64 {
    std::vector<unsigned long long> keys;
    std::vector<uint8_t> used;
    size_t mask;
    explicit HashSet64(size_t want)
    {
        size_t cap = 16;
        while (cap < 2 * want) cap <<= 1;
        keys.assign(cap, 0);
        used.assign(cap, 0);
        mask = cap - 1;
    }
    /* true when h was not present (and is now) */
    bool insert(unsigned long long h)
    {
        size_t i = (size_t)(h ^ (h >> 29)) & mask;
        while (used[i]) {
            if (keys[i] == h) return false;
            i = (i + 1) & mask;
        }
        used[i] = 1;
        keys[i] = h;
        return true;
    }
};

}  // namespace

extern "C" float rc_pool_vary(void *ctx, int which, int islands, int pop, int width,
                              const double *err, int nvars, int max_complexity, unsigned int seed,
                              unsigned int gen, int init_depth, int dedup, const unsigned int *ops,
                              int nops, const unsigned char *restart, const unsigned int *front,
                              const unsigned int *front_off, int nfront, double front_p,
                              unsigned short *out_len, unsigned short *out_cost,
                              unsigned long long *out_hash, double *out_err,
                              unsigned int *out_words)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !err || !ops || islands <= 0 || pop <= 0 || width < 2 || width > RV_WMAX) return -1.0f;
    if (nops <= 0 || nops > RV_MAXOPS || nvars < 0 || max_complexity < 0) return -1.0f;
    if (init_depth < 0 || init_depth > 15 || !(front_p >= 0.0)) return -1.0f;
    if (nfront < 0 || (nfront > 0 && (!front || !front_off))) return -1.0f;
    const int nslots = islands * pop;
    const int b = which & 1;
    if (nslots > c->pool_cap || width != c->pool_width || !c->d_pool[b] || !c->d_pool[b ^ 1])
        return -1.0f;
    RvConfig cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.width = width;
    cfg.nvars = nvars;
    cfg.max_complexity = max_complexity;
    cfg.init_depth = init_depth;
    cfg.dedup = dedup;
    cfg.seed = seed;
    cfg.gen = gen;
    cfg.islands = islands;
    cfg.pop = pop;
    cfg.nops = nops;
    bool nonterminal = false;
    for (int k = 0; k < nops; ++k) {
        const int a = (int)ops[2 * k + 1];
        if (a < 1 || a > 3 || rv_arity(ops[2 * k]) != a) return -1.0f;
        cfg.code[k] = ops[2 * k];
        cfg.by_arity[a][cfg.n_arity[a]++] = k;
        nonterminal = true;
    }
    if (!nonterminal) return -1.0f;
    cfg.nfront = front_p > 0.0 ? nfront : 0;
    cfg.front_p = front_p;
    const size_t nfw = cfg.nfront > 0 ? front_off[cfg.nfront] : 0;
    /* a front program must fit a slot, as FrontParents::from_front keeps only
       those (postfix.rs:369-383); the engine's buffers hold one slot */
    for (int f = 0; f < cfg.nfront; ++f)
        if (front_off[f + 1] < front_off[f] || front_off[f + 1] - front_off[f] > (unsigned)width ||
            front_off[f + 1] - front_off[f] < 2)
            return -1.0f;

    /* layout: inputs [err | restart | front | front_off], parent metadata,
       items, their programs, host programs and choices */
    const int nitems = nslots * RV_K;
    size_t cur = 0;
    const size_t o_err = rc_take(&cur, sizeof(double) * nslots);
    const size_t o_restart = rc_take(&cur, (size_t)islands);
    const size_t o_front = rc_take(&cur, sizeof(uint32_t) * (nfw + 1));
    const size_t o_foff = rc_take(&cur, sizeof(uint32_t) * (cfg.nfront + 1));
    const size_t in_end = rc_take(&cur, 0);
    const size_t o_plen = rc_take(&cur, sizeof(uint16_t) * nslots);
    const size_t o_pcost = rc_take(&cur, sizeof(int) * nslots);
    const size_t o_pcost16 = rc_take(&cur, sizeof(uint16_t) * nslots);
    const size_t o_phash = rc_take(&cur, sizeof(unsigned long long) * nslots);
    const size_t o_bad = rc_take(&cur, sizeof(int));
    const size_t o_items = rc_take(&cur, sizeof(RvItem) * nitems);
    const size_t meta_end = rc_take(&cur, 0);
    const size_t o_choice = rc_take(&cur, sizeof(RvChoice) * nslots);
    const size_t o_hprog = rc_take(&cur, sizeof(uint32_t) * (size_t)nslots * width);
    const size_t host_end = rc_take(&cur, 0);
    const size_t o_progs = rc_take(&cur, sizeof(uint32_t) * (size_t)nitems * width);
    const size_t dev_end = rc_take(&cur, 0);
    if (rc_reserve(c, dev_end, host_end) != 0) return -1.0f;
    unsigned char *dev = c->dev, *host = c->host;
    memcpy(host + o_err, err, sizeof(double) * nslots);
    for (int i = 0; i < islands; ++i) host[o_restart + i] = restart && restart[i] ? 1 : 0;
    if (nfw) memcpy(host + o_front, front, sizeof(uint32_t) * nfw);
    if (cfg.nfront) memcpy(host + o_foff, front_off, sizeof(uint32_t) * (cfg.nfront + 1));
    cudaEventRecord(c->t0, c->s);
    cudaMemcpyAsync(dev, host, in_end, cudaMemcpyHostToDevice, c->s);

    /* 1. parent metadata (read back with the items below: the tie-break and
       the elite) */
    uint16_t *d_plen = reinterpret_cast<uint16_t *>(dev + o_plen);
    int *d_pcost = reinterpret_cast<int *>(dev + o_pcost);
    uint16_t *d_pcost16 = reinterpret_cast<uint16_t *>(dev + o_pcost16);
    unsigned long long *d_phash = reinterpret_cast<unsigned long long *>(dev + o_phash);
    int *d_bad = reinterpret_cast<int *>(dev + o_bad);
    cudaMemsetAsync(d_bad, 0, sizeof(int), c->s);
    rv_parents<<<(nslots + RV_T - 1) / RV_T, RV_T, 0, c->s>>>(c->d_pool[b], width, nslots, d_plen,
                                                             d_pcost, d_pcost16, d_phash, d_bad);

    /* 2. the first RV_K attempts of every child slot */
    RvParents dpar;
    dpar.words = c->d_pool[b];
    dpar.err = reinterpret_cast<const double *>(dev + o_err);
    dpar.cost = d_pcost16;
    dpar.front = reinterpret_cast<const uint32_t *>(dev + o_front);
    dpar.front_off = reinterpret_cast<const uint32_t *>(dev + o_foff);
    RvItem *d_items = reinterpret_cast<RvItem *>(dev + o_items);
    uint32_t *d_progs = reinterpret_cast<uint32_t *>(dev + o_progs);
    rv_children<<<(nitems + RV_T - 1) / RV_T, RV_T, 0, c->s>>>(
        cfg, dpar, reinterpret_cast<const uint8_t *>(dev + o_restart), d_bad, d_items, d_progs);
    cudaMemcpyAsync(host + o_plen, dev + o_plen, meta_end - o_plen, cudaMemcpyDeviceToHost, c->s);
    c->launches += 2;
    if (rc_finish(c) != 0) return -1.0f;
    /* a parent slot that is not a valid program fails the call */
    if (*reinterpret_cast<const int *>(host + o_bad) != 0) return -1.0f;
    const uint16_t *cost16 = reinterpret_cast<const uint16_t *>(host + o_pcost16);

    /* 3. the duplicate rule, in slot order */
    const RvItem *items = reinterpret_cast<const RvItem *>(host + o_items);
    const unsigned long long *phash = reinterpret_cast<const unsigned long long *>(host + o_phash);
    const uint16_t *plen = reinterpret_cast<const uint16_t *>(host + o_plen);
    RvChoice *choice = reinterpret_cast<RvChoice *>(host + o_choice);
    uint32_t *hprog = reinterpret_cast<uint32_t *>(host + o_hprog);
    int nhost = 0;
    RvParents hpar;
    hpar.words = c->pool_host[b].data();
    hpar.err = err;
    hpar.cost = cost16;
    hpar.front = front;
    hpar.front_off = front_off;
    uint32_t prog[RV_WMAX], spans[RV_WMAX], other[RV_WMAX], tmp[RV_WMAX];
    auto host_program = [&](int n) {
        uint32_t *dst = hprog + (size_t)nhost * width;
        for (int q = 0; q < width; ++q) dst[q] = q < n ? prog[q] : RV_HALT;
        return nhost++;
    };
    HashSet64 seen((size_t)2 * nslots);
    if (dedup)
        for (int k = 0; k < nslots; ++k) seen.insert(phash[k]);
    for (int i = 0; i < islands; ++i) {
        const bool rs = restart && restart[i];
        int elite = i * pop;
        if (!rs) {
            RvKey kb = rv_key(err, cost16, elite);
            for (int k = i * pop + 1; k < (i + 1) * pop; ++k) {
                const RvKey kk = rv_key(err, cost16, k);
                if (rv_less(kk, kb)) {
                    elite = k;
                    kb = kk;
                }
            }
        }
        for (int j = 0; j < pop; ++j) {
            const int k = i * pop + j;
            RvChoice &ch = choice[k];
            ch.err = NAN;
            if (rs) {
                const RvItem &r = items[(size_t)k * RV_K];
                ch.src = RV_SRC_ITEM;
                ch.index = k * RV_K;
                ch.len = r.len;
                ch.cost = r.cost;
                ch.hash = r.hash;
                continue;
            }
            if (j == 0) {
                ch.src = RV_SRC_PARENT;
                ch.index = elite;
                ch.len = plen[elite];
                ch.cost = cost16[elite];
                ch.hash = phash[elite];
                ch.err = err[elite];
                continue;
            }
            bool done = false;
            for (int a = 0; a < 64 && !done; ++a) {
                int st, n = 0, cost = 0;
                uint64_t h = 0;
                if (a < RV_K) {
                    const RvItem &r = items[(size_t)k * RV_K + a];
                    st = r.status;
                    h = r.hash;
                    n = r.len;
                    cost = r.cost;
                } else {
                    st = rv_attempt(cfg, hpar, i, j, a, prog, &n, spans, other, tmp, &cost, &h);
                }
                if (st == RV_REJECT) continue;
                if (dedup && !seen.insert(h)) continue;
                if (st != RV_CANDIDATE) continue;
                if (a < RV_K) {
                    ch.src = RV_SRC_ITEM;
                    ch.index = k * RV_K + a;
                } else {
                    ch.src = RV_SRC_HOST;
                    ch.index = host_program(n);
                }
                ch.len = (uint16_t)n;
                ch.cost = (uint16_t)cost;
                ch.hash = h;
                done = true;
            }
            if (!done) {
                int n = 0, cost = 0;
                uint64_t h = 0;
                rv_random_slot(cfg, i, j, 64, prog, &n, spans, &cost, &h);
                ch.src = RV_SRC_HOST;
                ch.index = host_program(n);
                ch.len = (uint16_t)n;
                ch.cost = (uint16_t)cost;
                ch.hash = h;
            }
        }
    }

    /* 4. the children into the other pool */
    cudaMemcpyAsync(dev + o_choice, host + o_choice,
                    (o_hprog - o_choice) + sizeof(uint32_t) * (size_t)nhost * width,
                    cudaMemcpyHostToDevice, c->s);
    const size_t total = (size_t)nslots * width;
    const int grid = (int)std::min<size_t>((total + RV_T - 1) / RV_T, (size_t)c->sm_count * 16);
    rv_gather<<<grid, RV_T, 0, c->s>>>(width, nslots, reinterpret_cast<const RvChoice *>(dev + o_choice),
                                       d_progs, reinterpret_cast<const uint32_t *>(dev + o_hprog),
                                       c->d_pool[b], c->d_pool[b ^ 1]);
    c->launches += 1;
    cudaEventRecord(c->t1, c->s);
    /* the host mirror of the new pool, which the pool scorers read, and the
       caller's copy, both straight from the device */
    cudaMemcpyAsync(c->pool_host[b ^ 1].data(), c->d_pool[b ^ 1], sizeof(uint32_t) * total,
                    cudaMemcpyDeviceToHost, c->s);
    if (out_words)
        cudaMemcpyAsync(out_words, c->d_pool[b ^ 1], sizeof(uint32_t) * total,
                        cudaMemcpyDeviceToHost, c->s);
    if (rc_finish(c) != 0) return -1.0f;
    for (int k = 0; k < nslots; ++k) {
        if (out_len) out_len[k] = choice[k].len;
        if (out_cost) out_cost[k] = choice[k].cost;
        if (out_hash) out_hash[k] = choice[k].hash;
        if (out_err) out_err[k] = choice[k].err;
    }
    float ms = -1.0f;
    cudaEventElapsedTime(&ms, c->t0, c->t1);
    return ms;
}
