/*
 * Exact statistics over f64 predictions: rank-correlation sums
 * (eval.cu:2888-3133, :4093-4361), order statistics of |r|
 * (eval.cu:4365-4520, :4743-4850) and the maximum-error scan
 * (eval.cu:4522-4740).
 *
 * Rank sums. A (candidate, trial) segment's f64 predictions over all n rows
 * become order-preserving u64 keys (-0 folded onto +0, anything not finite
 * onto the largest key). Every position q needs its run [i, j) of equal keys
 * in sorted order, twice its centred average rank A = i + j - n, and the
 * exact sums sum A * B[row] and sum A^2 in 128-bit integers, B being the
 * target's own A. By default (up to 4,194,304 rows) the keys are cut into
 * buckets by splitters from a sorted sample and each bucket is ranked on its
 * own (the bucketed sums below). The radix path, which ranks the target once
 * per context, takes segments whose bucket overflows and serves the order
 * statistics, is a segmented LSD radix sort (8-bit digits, one kernel per
 * pass with decoupled look-back, a pass whose digit is constant over a
 * segment skipped) with the row as payload, then one pass over the sorted
 * keys for the runs. Integer sums do not depend on order, so either path is
 * bit-identical to the CPU's `RankTarget::sums` (metrics.rs:1359-1416) for
 * the same predictions.
 *
 * Order statistics sort the bit patterns of |pred - y| (non-negative, so
 * they order like the values) and pick the median or average the
 * interquartile window by rank. The maximum scan is an integer max over the
 * same patterns with the lowest attaining row, plus the per-row feasibility
 * interval of a level along one constant (reverse sweep for dr/dc).
 */
#include <algorithm>
#include <cstring>
#include <limits>
#include <vector>

#include "fit_common.cuh"
#include "fit_prep.h"
#include "rc_internal.h"
#include "rc_ops.cuh"

typedef unsigned long long u64;

#define RS_T 256                  /* sort / contribution threads */
#define RS_ITEMS 16               /* keys per thread */
#define RS_TILE (RS_T * RS_ITEMS) /* keys per tile */
#define RS_WARPS (RS_T / 32)
#define RK_T 256                  /* key threads (two rows each per step) */
#define RK_TILE 8192              /* rows per key block */
#define RK_WAVE_BYTES ((size_t)3 << 30)
#define RS_PASSES 8               /* 8-bit digits of a u64 key */

/* ---- keys -------------------------------------------------------------- */

/* Order-preserving key of an f64 (eval.cu:2921-2928 semantics): -0 shares
   +0's key, NaN is the largest key. */
__device__ __forceinline__ u64 rk_key(double v)
{
    if (v == 0.0) v = 0.0;
    if (isnan(v)) return ~0ULL;
    u64 b = (u64)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}

__device__ __forceinline__ u64 rk_abs_key(double r) { return (u64)__double_as_longlong(fabs(r)); }

__device__ __forceinline__ double rk_key_abs_value(u64 k) { return __longlong_as_double((long long)k); }

enum { RK_RANK = 0, RK_ABS = 1 };

/* Adds the counts of all eight digits of keys[r0, r1) to the block's
   shared table cnt[pass][digit]; all RS_T threads of the block call it. */
__device__ __forceinline__ void rs_count_keys(const u64 *src, long long r0, long long r1,
                                              unsigned int (*cnt)[256])
{
    const int tid = threadIdx.x, lane = tid & 31;
    for (long long c = r0; c < r1; c += 4 * RS_T) {
        /* four loads in flight per thread; every lane takes part in the
           warp votes, out-of-range ones with no digit */
        u64 k[4];
        bool in[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const long long idx = c + i * RS_T + tid;
            in[i] = idx < r1;
            k[i] = in[i] ? src[idx] : 0ULL;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int d = 0; d < RS_PASSES; ++d) {
                const unsigned dg = in[i] ? (unsigned)(k[i] >> (8 * d)) & 255u : 256u;
                /* a digit the whole warp shares (a constant segment, the
                   exponent bytes) is one add; the exponent bytes take few
                   values, so they are grouped; mantissa bytes scatter over
                   the bins and add one by one */
                if (__all_sync(0xffffffffu, dg == __shfl_sync(0xffffffffu, dg, 0))) {
                    if (lane == 0 && dg < 256u) atomicAdd(&cnt[d][dg], 32u);
                } else if (d >= 6) {
                    /* match_any here: this count is bound by its shared-memory
                       atomics, and the ballots' extra instructions cost more
                       than the match saves */
                    const unsigned peers = __match_any_sync(0xffffffffu, dg);
                    if (dg < 256u && lane == __ffs(peers) - 1)
                        atomicAdd(&cnt[d][dg], (unsigned)__popc(peers));
                } else if (dg < 256u) {
                    atomicAdd(&cnt[d][dg], 1u);
                }
            }
    }
}


/* Keys of segments [seg0, seg0 + gridDim.x / tiles) over all rows: the f64
   forward sweep of the segment's candidate at its constants
   (c0[seg * kmax + slot]), two rows per thread. RK_RANK keys the
   prediction; RK_ABS keys |pred - y| and flags a row whose prediction is
   not finite or exceeds 1e30 (eval.cu:4388-4418). A non-finite key marks
   the segment's status 2. The block then counts the eight digits of the
   keys it wrote (still in L2) into count[local segment][pass][256], which
   the caller zeroed, so the sort needs no counting read of its own (with
   count NULL it counts nothing). */
static_assert(RK_T == RS_T, "the digit count runs on the key kernel's blocks");
template <int MODE>
__global__ void __launch_bounds__(RK_T) rk_keys(const FIns *fins, const int *fins_off,
                                                const int4 *finfo, const int *valid,
                                                const double *c0, int kmax, const double *cols,
                                                const double *y, int npad, int n, int ntrials,
                                                int seg0, int tiles, int maxins, u64 *keys,
                                                unsigned int *rows, unsigned int *count,
                                                int *status)
{
    __shared__ unsigned int cnt[RS_PASSES][256];
    using V4 = FiV<double, 2>::V4;
    extern __shared__ __align__(16) unsigned char sm[];
    FIns *ins = reinterpret_cast<FIns *>(sm);
    double *cv = reinterpret_cast<double *>(sm + 8 * (size_t)((maxins + 1) & ~1));
    V4 *stk = reinterpret_cast<V4 *>(cv + FT_MAX_CONST);
    const int ls = blockIdx.x / tiles;
    const int seg = seg0 + ls;
    const int tile = blockIdx.x % tiles;
    const int cand = seg / ntrials;
    const int tid = threadIdx.x;
    const bool ok = valid[cand] != 0;
    const int nf = finfo[cand].x;
#pragma unroll
    for (int d = 0; d < RS_PASSES; ++d) cnt[d][tid] = 0;
    if (ok) {
        for (int i = tid; i < nf; i += RK_T) ins[i] = fins[fins_off[cand] + i];
        if (tid < FT_MAX_CONST) cv[tid] = tid < kmax ? c0[(size_t)seg * kmax + tid] : 0.0;
    }
    __syncthreads();
    const int r0 = tile * RK_TILE, r1 = min(n, r0 + RK_TILE);
    u64 *kseg = keys + (size_t)ls * n;
    unsigned int *rseg = rows ? rows + (size_t)ls * n : nullptr;
    bool bad = !ok;
    for (int row = r0 + 2 * tid; row < r1; row += 2 * RK_T) {
        double pr[2] = {CUDART_NAN, CUDART_NAN};
        if (ok) fi_forward<double, 2, false>(ins, cv, cols, npad, row, stk, nullptr, RK_T, tid, pr);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int rr = row + i;
            if (rr >= r1) continue;
            u64 k;
            if (MODE == RK_RANK) {
                if (!isfinite(pr[i])) {
                    k = ~0ULL;
                    bad = true;
                } else {
                    k = rk_key(pr[i]);
                }
            } else {
                const double r = pr[i] - y[rr];
                if (!isfinite(pr[i]) || fabs(pr[i]) > 1e30 || !isfinite(r)) {
                    k = ~0ULL;
                    bad = true;
                } else {
                    k = rk_abs_key(r);
                }
            }
            kseg[rr] = k;
            if (rseg) rseg[rr] = (unsigned int)rr;
        }
    }
    /* (the barrier also makes the block's key writes visible to its reads) */
    if (__syncthreads_or(bad) && tid == 0) status[seg] = 2;
    if (!count) return; /* the bucketed sums count nothing here */
    rs_count_keys(kseg, r0, r1, cnt);
    __syncthreads();
#pragma unroll
    for (int d = 0; d < RS_PASSES; ++d)
        if (cnt[d][tid]) atomicAdd(&count[((size_t)ls * RS_PASSES + d) * 256 + tid], cnt[d][tid]);
}

/* Keys of the target (one segment). */
__global__ void rk_target_keys(const double *y, int n, u64 *keys, unsigned int *rows)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        keys[i] = rk_key(y[i]);
        rows[i] = (unsigned int)i;
    }
}

/* ---- segmented LSD radix sort (one sweep per digit) ---------------------
 * Keys are u64, 8-bit digits, up to eight passes. One read of the keys first
 * counts every digit of every pass per segment (rs_count); rs_prep turns the
 * counts into each digit's first output position, marks the passes whose
 * digit is constant over a segment (they leave the order unchanged and are
 * skipped) and which buffer ends up holding each segment. A pass is then one
 * kernel (rs_pass): every tile ranks its keys by digit, publishes its digit
 * counts, adds up its predecessors' counts by decoupled look-back over the
 * published words, and writes its keys to their final places of the pass.
 * Tiles take increasing tickets per pass (segments interleaved), so every
 * tile a tile waits on has started before it; each wait is bounded, and a
 * wait that gives up raises a flag that stops every other wait and every
 * write, and fails the call. */

#define RS_ST_AGG 1ULL    /* published word: the tile's own counts */
#define RS_ST_PREFIX 2ULL /* published word: counts of this and every earlier tile */
#define RS_SPIN_LIMIT (1u << 22)

/* A published look-back word: kind in bits 62-63, pass tag (1-8) in bits
   32-39, the count in bits 0-31. Words of another pass read as unpublished. */
__device__ __forceinline__ u64 rs_word(u64 kind, int pass, unsigned int v)
{
    return (kind << 62) | ((u64)(pass + 1) << 32) | (u64)v;
}

/* Lanes of the warp holding the same 9-bit label (a digit, or 256 for a lane
   with no key): one ballot per bit, each lane keeping the lanes that agree
   with it on that bit. The same mask as __match_any_sync on the label, from
   nine votes. */
__device__ __forceinline__ unsigned rs_peers(unsigned d)
{
    unsigned m = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < 9; ++b) {
        const bool bit = (d >> b) & 1u;
        const unsigned v = __ballot_sync(0xffffffffu, bit);
        m &= bit ? v : ~v;
    }
    return m;
}

/* Per segment, the counts of all eight digits: count[seg][pass][256]. A
   block counts RS_COUNT_TILES tiles in shared memory before adding to the
   segment's totals. */
#define RS_COUNT_TILES 8
__global__ void __launch_bounds__(RS_T) rs_count(const u64 *keys, int n, int nblk,
                                                 unsigned int *count)
{
    __shared__ unsigned int cnt[RS_PASSES][256];
    const int seg = blockIdx.x / nblk, blk = blockIdx.x % nblk;
    const int tid = threadIdx.x;
    const u64 *src = keys + (size_t)seg * n;
#pragma unroll
    for (int d = 0; d < RS_PASSES; ++d) cnt[d][tid] = 0;
    __syncthreads();
    const long long r0 = (long long)blk * RS_COUNT_TILES * RS_TILE;
    const long long r1 = min((long long)n, r0 + (long long)RS_COUNT_TILES * RS_TILE);
    rs_count_keys(src, r0, r1, cnt);
    __syncthreads();
#pragma unroll
    for (int d = 0; d < RS_PASSES; ++d)
        if (cnt[d][tid]) atomicAdd(&count[((size_t)seg * RS_PASSES + d) * 256 + tid], cnt[d][tid]);
}

/* Per segment: digit counts -> first output positions (in place), the mask
   of skipped passes, and the buffer that holds the sorted keys. */
__global__ void __launch_bounds__(256) rs_prep(unsigned int *count, int n, unsigned char *skip,
                                               unsigned char *par)
{
    __shared__ unsigned int wsum[8];
    const int seg = blockIdx.x, d = threadIdx.x, lane = d & 31, w = d >> 5;
    unsigned mask = 0;
    for (int pass = 0; pass < RS_PASSES; ++pass) {
        unsigned int *h = count + ((size_t)seg * RS_PASSES + pass) * 256;
        const unsigned int total = h[d];
        unsigned int x = total;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        const int all = __syncthreads_or(total == (unsigned)n);
        unsigned int before = 0;
        for (int k = 0; k < w; ++k) before += wsum[k];
        h[d] = before + x - total;
        if (all) mask |= 1u << pass;
        __syncthreads();
    }
    if (d == 0) {
        skip[seg] = (unsigned char)mask;
        par[seg] = (unsigned char)(__popc(~mask & 0xffu) & 1);
    }
}

/* One pass over every segment's tiles. Warp w ranks its keys among the
   warp's earlier keys of the same digit (a peer mask per round of 32); the
   warps' counts are scanned in warp order, so the pass is stable. The tile
   is reordered by digit in shared memory first, so that consecutive threads
   write consecutive addresses of each digit's output run. Keys and then row
   payloads go through the same 32 KB stage: between the two, each thread
   keeps its keys' slots in the digit-ordered tile and the output positions
   of the slots it wrote, so four blocks share an SM. */
template <bool VALS>
__host__ __device__ constexpr size_t rs_pass_smem()
{
    return sizeof(u64) * RS_TILE;
}

template <bool VALS>
__global__ void __launch_bounds__(RS_T, 4) rs_pass(u64 *ka, u64 *kb, unsigned int *va,
                                                   unsigned int *vb, const unsigned char *skip,
                                                   const unsigned int *goff_all, u64 *state,
                                                   int *ticket, int *abort_flag, int n,
                                                   int ntiles, int pass)
{
    extern __shared__ __align__(16) unsigned char sm[];
    u64 *skey = reinterpret_cast<u64 *>(sm);
    unsigned int *sval = reinterpret_cast<unsigned int *>(sm);
    __shared__ unsigned int cnt[RS_WARPS][256];
    __shared__ unsigned int gdelta[256], wsum[RS_WARPS];
    __shared__ int s_ticket;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) s_ticket = atomicAdd(ticket + pass, 1);
    __syncthreads();
    /* segments interleave in ticket order, so the tiles in flight spread
       over the segments and each look-back chain stays short */
    const int nseg = (int)(gridDim.x / (unsigned)ntiles);
    const int seg = s_ticket % nseg, tile = s_ticket / nseg;
    const unsigned mask = skip[seg];
    if (mask & (1u << pass)) return;
    const int shift = 8 * pass;
    const bool p = (__popc(~mask & ((1u << pass) - 1u)) & 1) != 0;
    const size_t sb = (size_t)seg * n;
    const u64 *src = (p ? kb : ka) + sb;
    u64 *dst = (p ? ka : kb) + sb;
    const unsigned int *vsrc = VALS ? (p ? vb : va) + sb : nullptr;
    unsigned int *vdst = VALS ? (p ? va : vb) + sb : nullptr;
#pragma unroll
    for (int k = 0; k < RS_WARPS; ++k) cnt[k][tid] = 0;
    constexpr int R = RS_TILE / RS_WARPS / 32;
    static_assert(R == RS_ITEMS, "a thread stages as many keys as it writes");
    const int t0 = tile * RS_TILE;
    const int wb = w * (RS_TILE / RS_WARPS);
    const int count = min(RS_TILE, n - t0);
    const unsigned lt = (1u << lane) - 1u;
    u64 key[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int li = wb + 32 * r + lane;
        key[r] = li < count ? src[t0 + li] : 0ULL;
    }
    __syncthreads();
    /* rank of key r among the tile's earlier keys of its digit, two 16-bit
       halves per register (ranks and slots are below RS_TILE) */
    unsigned int rk[R / 2];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const bool in = wb + 32 * r + lane < count;
        const unsigned d = in ? (unsigned)(key[r] >> shift) & 255u : 256u;
        const unsigned peers = rs_peers(d);
        const unsigned int base = in ? cnt[w][d] : 0u;
        const unsigned int rr = base + __popc(peers & lt);
        rk[r / 2] = (r & 1) ? (rk[r / 2] | (rr << 16)) : rr;
        __syncwarp();
        if (in && lane == __ffs(peers) - 1) cnt[w][d] = base + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    /* per digit (thread tid): warp prefixes and the tile's count */
    unsigned int tot = 0;
#pragma unroll
    for (int k = 0; k < RS_WARPS; ++k) {
        const unsigned int c = cnt[k][tid];
        cnt[k][tid] = tot;
        tot += c;
    }
    /* publish the tile's counts at once, for the tiles that look back on it */
    volatile u64 *st = reinterpret_cast<volatile u64 *>(state) + (size_t)seg * ntiles * 256;
    st[(size_t)tile * 256 + tid] = rs_word(tile == 0 ? RS_ST_PREFIX : RS_ST_AGG, pass, tot);
    /* the tile's digit starts in the digit-ordered tile */
    unsigned int x = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    unsigned int before = 0;
    for (int k = 0; k < w; ++k) before += wsum[k];
    /* digit tid starts at ls in the digit-ordered tile; cnt[k][tid] becomes
       the slot of warp k's first key of that digit */
    const unsigned int ls = before + x - tot;
#pragma unroll
    for (int k = 0; k < RS_WARPS; ++k) cnt[k][tid] += ls;
    /* slot i of digit d goes to gdelta[d] + i (mod 2^32), once the earlier
       tiles' counts (excl) are added below */
    gdelta[tid] = goff_all[((size_t)seg * RS_PASSES + pass) * 256 + tid] - ls;
    __syncthreads();
    /* keys into the stage; key r's rank becomes its slot there (< count) */
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int li = wb + 32 * r + lane;
        if (li >= count) continue;
        const unsigned d = (unsigned)(key[r] >> shift) & 255u;
        const unsigned int lp = cnt[w][d] + ((rk[r / 2] >> (16 * (r & 1))) & 0xffffu);
        skey[lp] = key[r];
        rk[r / 2] = (r & 1) ? ((rk[r / 2] & 0xffffu) | (lp << 16)) : ((rk[r / 2] & 0xffff0000u) | lp);
    }
    /* look back over the earlier tiles of the segment */
    unsigned int excl = 0;
    bool failed = false;
    for (int j = tile - 1; j >= 0 && !failed; --j) {
        unsigned spins = 0, ns = 8;
        u64 v;
        for (;;) {
            v = st[(size_t)j * 256 + tid];
            if ((int)((v >> 32) & 0xffu) == pass + 1 && (v >> 62) != 0) break;
            if (++spins > RS_SPIN_LIMIT || *(volatile int *)abort_flag) {
                atomicExch(abort_flag, 1);
                failed = true;
                break;
            }
            __nanosleep(ns);
            if (ns < 256) ns <<= 1;
        }
        if (failed) break;
        excl += (unsigned int)v;
        if ((v >> 62) == RS_ST_PREFIX) break;
    }
    if (tile > 0 && !failed)
        st[(size_t)tile * 256 + tid] = rs_word(RS_ST_PREFIX, pass, excl + tot);
    gdelta[tid] += excl;
    if (__syncthreads_or(failed)) return;
    /* slot i = tid + k * RS_T leaves for its output position pos[k] */
    unsigned int pos[RS_ITEMS];
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const int i = tid + k * RS_T;
        pos[k] = 0xffffffffu;
        if (i >= count) continue;
        const u64 kk = skey[i];
        const unsigned d = (unsigned)(kk >> shift) & 255u;
        const unsigned int q = gdelta[d] + (unsigned)i;
        if (q >= (unsigned)n) {
            atomicExch(abort_flag, 1);
            continue;
        }
        dst[q] = kk;
        pos[k] = q;
    }
    if (!VALS) return;
    __syncthreads(); /* every key has left the stage */
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int li = wb + 32 * r + lane;
        if (li < count) sval[(rk[r / 2] >> (16 * (r & 1))) & 0xffffu] = vsrc[t0 + li];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k)
        if (pos[k] != 0xffffffffu) vdst[pos[k]] = sval[tid + k * RS_T];
}

struct RsBuffers {
    u64 *ka, *kb;
    unsigned int *va, *vb;
    unsigned int *count; /* [nseg][8][256] digit counts, then first positions */
    u64 *state;          /* [nseg][ntiles][256] look-back words */
    int *ticket;         /* [8] per-pass tile tickets */
    unsigned char *par, *skip;
};

/* Sort `nseg` segments of n keys (with row payloads when VALS) across the
   two buffers; par[seg] tells which holds the result. Returns the number of
   kernels launched. A look-back that gave up, or a position out of range,
   sets *abort_flag (which the caller zeroes once and checks after). */
template <bool VALS>
unsigned long long rs_sort(const RsBuffers &b, int nseg, int n, int *abort_flag, cudaStream_t s,
                           bool counted)
{
    const int ntiles = (n + RS_TILE - 1) / RS_TILE;
    const int nblk = (ntiles + RS_COUNT_TILES - 1) / RS_COUNT_TILES;
    rc_raise_smem((const void *)rs_pass<VALS>, rs_pass_smem<VALS>());
    cudaMemsetAsync(b.state, 0, sizeof(u64) * 256 * (size_t)ntiles * (size_t)nseg, s);
    cudaMemsetAsync(b.ticket, 0, sizeof(int) * RS_PASSES, s);
    if (!counted) {
        cudaMemsetAsync(b.count, 0, sizeof(unsigned int) * RS_PASSES * 256 * (size_t)nseg, s);
        rs_count<<<(unsigned)nseg * (unsigned)nblk, RS_T, 0, s>>>(b.ka, n, nblk, b.count);
    }
    rs_prep<<<nseg, 256, 0, s>>>(b.count, n, b.skip, b.par);
    const unsigned grid = (unsigned)nseg * (unsigned)ntiles;
    for (int pass = 0; pass < RS_PASSES; ++pass)
        rs_pass<VALS><<<grid, RS_T, rs_pass_smem<VALS>(), s>>>(
            b.ka, b.kb, b.va, b.vb, b.skip, b.count, b.state, b.ticket, abort_flag, n, ntiles,
            pass);
    return (counted ? 1 : 2) + RS_PASSES;
}

/* ---- runs and exact sums ----------------------------------------------- */

/* Block exclusive max (forward) of an int over the 256 threads. */
__device__ __forceinline__ int rk_excl_max(int v, int *sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = max(x, y);
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    int before = -1;
    for (int k = 0; k < w; ++k) before = max(before, sh[k]);
    int ex = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) ex = -1;
    __syncthreads();
    return max(before, ex);
}

/* Block exclusive min from the right of an int over the 256 threads. */
__device__ __forceinline__ int rk_excl_min_right(int v, int *sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_down_sync(0xffffffffu, x, o);
        if (lane + o < 32) x = min(x, y);
    }
    if (lane == 0) sh[w] = x;
    __syncthreads();
    int after = 0x7fffffff;
    for (int k = w + 1; k < RS_WARPS; ++k) after = min(after, sh[k]);
    int ex = __shfl_down_sync(0xffffffffu, x, 1);
    if (lane == 31) ex = 0x7fffffff;
    __syncthreads();
    return min(after, ex);
}

/* First index in [lo, hi) whose key is >= k (keys sorted). */
__device__ int rk_lower(const u64 *keys, int lo, int hi, u64 k)
{
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (keys[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

/* First index in [lo, hi) whose key is > k (keys sorted), or hi. */
__device__ int rk_upper(const u64 *keys, int lo, int hi, u64 k)
{
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (keys[mid] <= k) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

enum { RK_SUMS = 0, RK_FILL = 1 };

/* Sum of a 128-bit integer over the block's RS_T threads (a tree in shared
   memory; integers, so exact in any order). Every thread gets the sum. */
__device__ __forceinline__ __int128 rk_block_sum(__int128 v, __int128 *red)
{
    const int tid = threadIdx.x;
    red[tid] = v;
    __syncthreads();
#pragma unroll
    for (int h = RS_T / 2; h > 0; h >>= 1) {
        if (tid < h) red[tid] += red[tid + h];
        __syncthreads();
    }
    const __int128 s = red[0];
    __syncthreads();
    return s;
}

/* One tile of a sorted segment: every position's run [i, j) (block scans
   of the run starts inside the tile; a binary search for a run that crosses
   the tile's edge), A = i + j - n, and the tile's exact partial sums.
   RK_SUMS: part = (sum A * B[row], sum A^2). RK_FILL (the target): B[row] = A
   and part = (0, sum A^2). */
template <int MODE>
__global__ void __launch_bounds__(RS_T) rk_runs(const u64 *ka, const u64 *kb,
                                                const unsigned int *va, const unsigned int *vb,
                                                const unsigned char *par, int n, int ntiles,
                                                const long long *B, long long *Bout,
                                                __int128 *part)
{
    __shared__ int sh[RS_WARPS];
    __shared__ int s_left, s_right;
    __shared__ __int128 red[RS_T];
    const int seg = blockIdx.x / ntiles, tile = blockIdx.x % ntiles;
    const int tid = threadIdx.x;
    const size_t sb = (size_t)seg * n;
    const bool p = par[seg] != 0;
    const u64 *keys = (p ? kb : ka) + sb;
    const unsigned int *vals = (p ? vb : va) + sb;
    const int t0 = tile * RS_TILE, t1 = min(n, t0 + RS_TILE);
    const int q0 = t0 + tid * RS_ITEMS;
    u64 k[RS_ITEMS];
    bool f[RS_ITEMS];
    u64 prev = (q0 > 0 && q0 < t1) ? keys[q0 - 1] : 0ULL;
    int last = -1, first = 0x7fffffff;
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {
        const int q = q0 + j;
        const bool in = q < t1;
        k[j] = in ? keys[q] : 0ULL;
        f[j] = in && (q == 0 || k[j] != prev);
        prev = k[j];
        if (f[j]) {
            last = q;
            first = min(first, q);
        }
    }
    if (tid == 0) {
        /* the run holding the tile's first position may start earlier; the
           one holding its last position may end later */
        const u64 kf = keys[t0], kl = keys[t1 - 1];
        s_left = (t0 > 0 && keys[t0 - 1] == kf) ? rk_lower(keys, 0, t0, kf) : t0;
        s_right = (t1 < n && keys[t1] == kl) ? rk_upper(keys, t1, n, kl) : t1;
    }
    const int ex_start = rk_excl_max(last, sh);
    const int ex_end = rk_excl_min_right(first, sh);
    const int start0 = ex_start >= 0 ? ex_start : s_left;
    int end = ex_end != 0x7fffffff ? ex_end : s_right;
    int st[RS_ITEMS];
    {
        int cur = start0;
#pragma unroll
        for (int j = 0; j < RS_ITEMS; ++j) {
            if (f[j]) cur = q0 + j;
            st[j] = cur;
        }
    }
    __int128 ab = 0, aa = 0;
#pragma unroll
    for (int j = RS_ITEMS - 1; j >= 0; --j) {
        const int q = q0 + j;
        if (q < t1) {
            const long long A = (long long)st[j] + (long long)end - (long long)n;
            const unsigned int row = vals[q];
            aa += (__int128)A * A;
            if (MODE == RK_SUMS) ab += (__int128)A * B[row];
            else Bout[row] = A;
            if (f[j]) end = q;
        }
    }
    const __int128 sab = rk_block_sum(ab, red);
    const __int128 saa = rk_block_sum(aa, red);
    if (tid == 0) {
        part[((size_t)seg * ntiles + tile) * 2 + 0] = sab;
        part[((size_t)seg * ntiles + tile) * 2 + 1] = saa;
    }
}

/* One block per segment: the tile partials summed into two 128-bit values,
   written as (hi, lo) u64 pairs at out[4 * seg ...] (two's complement). */
__global__ void __launch_bounds__(RS_T) rk_final(const __int128 *part, int ntiles, u64 *out)
{
    __shared__ __int128 red[RS_T];
    const int seg = blockIdx.x, tid = threadIdx.x;
    __int128 ab = 0, aa = 0;
    for (int t = tid; t < ntiles; t += RS_T) {
        ab += part[((size_t)seg * ntiles + t) * 2 + 0];
        aa += part[((size_t)seg * ntiles + t) * 2 + 1];
    }
    const unsigned __int128 uab = (unsigned __int128)rk_block_sum(ab, red);
    const unsigned __int128 uaa = (unsigned __int128)rk_block_sum(aa, red);
    if (tid == 0) {
        out[(size_t)seg * 4 + 0] = (u64)(uab >> 64);
        out[(size_t)seg * 4 + 1] = (u64)uab;
        out[(size_t)seg * 4 + 2] = (u64)(uaa >> 64);
        out[(size_t)seg * 4 + 3] = (u64)uaa;
    }
}

/* ---- bucketed rank sums -------------------------------------------------
 *
 * The sums need every key's run [i, j) of equal keys in sorted order, not the
 * sorted array. So a segment is cut into buckets that are ordered among
 * themselves: splitters taken from a sorted sample of its keys (RB_OVS
 * samples per bucket, from rows spread over the segment by a fixed hash)
 * give a range bucket between consecutive splitters and an equality bucket
 * for each splitter. One pass puts every key of a range bucket, with its
 * row's B, into the bucket's fixed-capacity slots (block-aggregated
 * reservations); a key equal to a splitter only adds to its equality
 * bucket's count and B sum. A scan per segment gives every bucket its first
 * position. One block per range bucket then groups its keys by a 10-bit
 * digit of their offset from the bucket's smallest key, scaled to the bits
 * that vary inside the bucket: a group of equal keys is one run, and a small
 * group of distinct keys ranks each key by comparison; a bucket with a large
 * group of distinct keys is sorted in shared memory instead. A bucket over
 * its capacity sends the whole segment to the radix sort above. The sums are
 * integers, so they are the same bits on every path. */
#define RB_AVG 2048                /* keys per range bucket aimed at */
#define RB_CAP 8192                /* slots per range bucket */
#define RB_OVS 8                   /* samples per range bucket */
#define RB_MAXB 2048               /* range buckets per segment at most */
#define RB_MAXS (RB_OVS * RB_MAXB) /* samples per segment at most (a power of two) */
#define RB_DIG 1024                /* digit groups of a range bucket */
#define RB_GMAX 48                 /* largest group of distinct keys ranked by comparison */
static_assert((RB_CAP & (RB_CAP - 1)) == 0, "a sorted bucket pads to a power of two");
#define RB_CT 4096                 /* keys per scatter block */
#define RB_CTT 256                 /* scatter threads */
#define RB_CR (RB_CT / RB_CTT)
#define RB_ST 1024 /* splitter and scan threads */
static_assert(RB_CT <= 65536 && 2 * RB_MAXB <= 65536, "bucket and rank pack into 16 bits each");

__device__ __forceinline__ unsigned rb_hash(unsigned a, unsigned b)
{
    unsigned h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u);
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

/* Keys of S sample rows per segment: S / 2 row pairs, pair p at rows 2q and
   2q + 1 with q drawn by a fixed hash from the p-th of S / 2 equal strata of
   the n / 2 pairs; the f64 sweep and the keys of rk_keys. */
__global__ void __launch_bounds__(RK_T) rb_sample(const FIns *fins, const int *fins_off,
                                                  const int4 *finfo, const int *valid,
                                                  const double *c0, int kmax, const double *cols,
                                                  int npad, int n, int ntrials, int seg0,
                                                  int sblocks, int S, int maxins, u64 *samp)
{
    using V4 = FiV<double, 2>::V4;
    extern __shared__ __align__(16) unsigned char sm[];
    FIns *ins = reinterpret_cast<FIns *>(sm);
    double *cv = reinterpret_cast<double *>(sm + 8 * (size_t)((maxins + 1) & ~1));
    V4 *stk = reinterpret_cast<V4 *>(cv + FT_MAX_CONST);
    const int ls = blockIdx.x / sblocks, blk = blockIdx.x % sblocks;
    const int seg = seg0 + ls;
    const int cand = seg / ntrials;
    const int tid = threadIdx.x;
    const bool ok = valid[cand] != 0;
    if (ok) {
        const int nf = finfo[cand].x;
        for (int i = tid; i < nf; i += RK_T) ins[i] = fins[fins_off[cand] + i];
        if (tid < FT_MAX_CONST) cv[tid] = tid < kmax ? c0[(size_t)seg * kmax + tid] : 0.0;
    }
    __syncthreads();
    const int hp = S / 2, p = blk * RK_T + tid;
    if (p >= hp) return;
    const int stride = (n / 2) / hp;
    const int q = p * stride + (int)(rb_hash((unsigned)seg, (unsigned)p) % (unsigned)stride);
    double pr[2] = {CUDART_NAN, CUDART_NAN};
    if (ok) fi_forward<double, 2, false>(ins, cv, cols, npad, 2 * q, stk, nullptr, RK_T, tid, pr);
#pragma unroll
    for (int i = 0; i < 2; ++i)
        samp[(size_t)ls * RB_MAXS + 2 * p + i] = isfinite(pr[i]) ? rk_key(pr[i]) : ~0ULL;
}

/* One block per segment: the S samples sorted (bitonic, padded to P2 with the
   largest key), splitter j = sample (j + 1) * S / m for j < m - 1 with
   repeats dropped, into spl[seg][..] and their count into nspl[seg]. */
__global__ void __launch_bounds__(RB_ST) rb_splitters(const u64 *samp, int S, int P2, int m,
                                                      u64 *spl, int *nspl)
{
    extern __shared__ __align__(16) unsigned char sm[];
    u64 *s = reinterpret_cast<u64 *>(sm);
    const int ls = blockIdx.x, tid = threadIdx.x;
    const u64 *src = samp + (size_t)ls * RB_MAXS;
    for (int i = tid; i < P2; i += RB_ST) s[i] = i < S ? src[i] : ~0ULL;
    __syncthreads();
    for (int k = 2; k <= P2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < P2; i += RB_ST) {
                const int l = i ^ j;
                if (l > i) {
                    const u64 a = s[i], b = s[l];
                    if ((a > b) == ((i & k) == 0)) {
                        s[i] = b;
                        s[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    if (tid < 32) {
        int cnt = 0;
        for (int j0 = 0; j0 < m - 1; j0 += 32) {
            const int j = j0 + tid;
            u64 v = 0;
            bool keep = false;
            if (j < m - 1) {
                v = s[(j + 1) * S / m];
                keep = j == 0 || v != s[j * S / m];
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (keep) spl[(size_t)ls * RB_MAXB + cnt + __popc(bal & ((1u << tid) - 1u))] = v;
            cnt += __popc(bal);
        }
        if (tid == 0) nspl[ls] = cnt;
    }
}

/* RB_CT keys per block: each key's bucket, the block's count per bucket (a
   key's rank among the block's keys of its bucket from the shared-memory
   count), one reservation per range bucket the block touches, then the
   range keys and their B written to their slots. Equality buckets only add
   counts and B sums. A slot at or past `cap` flags the segment. */
__global__ void __launch_bounds__(RB_CTT, 3) rb_scatter(const u64 *keys, int n, int ctiles, int m,
                                                   int cap, const long long *B, const u64 *spl,
                                                   const int *nspl, unsigned *rcur,
                                                   unsigned *ecnt, unsigned long long *esum,
                                                   u64 *bkey, int *bval, int *ovf)
{
    __shared__ u64 sspl[RB_MAXB];
    __shared__ unsigned hist[2 * RB_MAXB];
    __shared__ unsigned long long ssum[RB_MAXB];
    const int ls = blockIdx.x / ctiles, tile = blockIdx.x % ctiles, tid = threadIdx.x;
    const int ns = nspl[ls], nb = 2 * ns + 1;
    for (int i = tid; i < ns; i += RB_CTT) {
        sspl[i] = spl[(size_t)ls * RB_MAXB + i];
        ssum[i] = 0ULL;
    }
    for (int i = tid; i < nb; i += RB_CTT) hist[i] = 0u;
    __syncthreads();
    const u64 *ks = keys + (size_t)ls * n;
    const int t0 = tile * RB_CT;
    /* every key and its B loaded first, then all of them searched a level at
       a time (the lower bound among the splitters by binary lifting), so
       the loads and the shared-memory probes overlap */
    u64 key[RB_CR];
    int bv[RB_CR];
    unsigned pk[RB_CR];
#pragma unroll
    for (int r = 0; r < RB_CR; ++r) {
        const int i = t0 + r * RB_CTT + tid;
        const bool in = i < n;
        key[r] = in ? ks[i] : 0ULL;
        bv[r] = in ? (int)B[i] : 0;
        pk[r] = 0u;
    }
    int top = 1;
    while (top <= ns) top <<= 1;
    for (int step = top >> 1; step > 0; step >>= 1) {
#pragma unroll
        for (int r = 0; r < RB_CR; ++r) {
            const unsigned p = pk[r] + (unsigned)step;
            if (p <= (unsigned)ns && sspl[p - 1] < key[r]) pk[r] = p;
        }
    }
#pragma unroll
    for (int r = 0; r < RB_CR; ++r) {
        if (t0 + r * RB_CTT + tid >= n) {
            pk[r] = 0xffffffffu;
            continue;
        }
        const unsigned p = pk[r];
        const bool eq = p < (unsigned)ns && sspl[p] == key[r];
        const unsigned b = 2u * p + (eq ? 1u : 0u);
        const unsigned rank = atomicAdd(&hist[b], 1u);
        if (eq) atomicAdd(&ssum[p], (unsigned long long)(long long)bv[r]);
        pk[r] = (b << 16) | rank;
    }
    __syncthreads();
    for (int b = tid; b < nb; b += RB_CTT) {
        const unsigned h = hist[b];
        if (!h) continue;
        const size_t j = (size_t)ls * RB_MAXB + (b >> 1);
        if (b & 1) {
            atomicAdd(&ecnt[j], h);
            atomicAdd(&esum[j], ssum[b >> 1]);
        } else {
            hist[b] = atomicAdd(&rcur[j], h);
        }
    }
    __syncthreads();
    bool over = false;
#pragma unroll
    for (int r = 0; r < RB_CR; ++r) {
        if (pk[r] == 0xffffffffu) continue;
        const unsigned b = pk[r] >> 16;
        if (b & 1u) continue;
        const unsigned pos = hist[b] + (pk[r] & 0xffffu);
        if (pos >= (unsigned)cap) {
            over = true;
            continue;
        }
        const size_t slot = ((size_t)ls * m + (b >> 1)) * RB_CAP + pos;
        bkey[slot] = key[r];
        bval[slot] = bv[r];
    }
    if (over) ovf[ls] = 1;
}

/* One block per segment: bucket sizes in order (range 0, equality 0, range
   1, ...), their first positions, and the equality buckets' partial sums
   (one run [O, O + c) each: A = 2 O + c - n). A range bucket over `cap`, or
   sizes that do not add up to n, flag the segment. */
__global__ void __launch_bounds__(RB_ST) rb_scan(int n, int cap, const int *nspl,
                                                 const unsigned *rcur, const unsigned *ecnt,
                                                 const unsigned long long *esum, unsigned *boff,
                                                 __int128 *part, int *ovf)
{
    __shared__ unsigned wsum[RB_ST / 32];
    const int ls = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int nb = 2 * nspl[ls] + 1;
    unsigned sz[4], tot = 0;
    bool bad = false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int b = 4 * tid + k;
        unsigned v = 0;
        if (b < nb) {
            const size_t j = (size_t)ls * RB_MAXB + (b >> 1);
            v = (b & 1) ? ecnt[j] : rcur[j];
            if (!(b & 1) && v > (unsigned)cap) bad = true;
        }
        sz[k] = v;
        tot += v;
    }
    unsigned x = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    unsigned run = x - tot;
    for (int k = 0; k < w; ++k) run += wsum[k];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int b = 4 * tid + k;
        if (b < nb) {
            const size_t e = (size_t)ls * 2 * RB_MAXB + b;
            boff[e] = run;
            if (b & 1) {
                const long long c = sz[k];
                const long long A = 2LL * run + c - n;
                const long long sb = (long long)esum[(size_t)ls * RB_MAXB + (b >> 1)];
                part[e * 2 + 0] = (__int128)A * sb;
                part[e * 2 + 1] = (__int128)c * A * A;
            }
        }
        run += sz[k];
    }
    if (tid == RB_ST - 1 && run != (unsigned)n) bad = true;
    if (bad) ovf[ls] = 1;
}

/* Shared layout of rb_local: the bucket's keys and B in digit order, the
   digit groups' first positions (RB_DIG + 1), their cursors and flags. */
__host__ __device__ constexpr size_t rb_local_smem()
{
    return (size_t)RB_CAP * (sizeof(u64) + sizeof(int)) + (2 * RB_DIG + 1) * sizeof(unsigned) +
           RB_DIG;
}

/* Sum of a 64-bit integer over a block of NT threads: warp butterflies, then
   warp partials in order (integers: exact in any order). Every thread gets
   the sum; `ws` holds NT / 32 values. */
template <int NT>
__device__ __forceinline__ long long rb_block_sum64(long long v, long long *ws)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    long long s = 0;
#pragma unroll
    for (int k = 0; k < NT / 32; ++k) s += ws[k];
    __syncthreads();
    return s;
}

#define RB_LT 512 /* rb_local threads */
static_assert(RB_DIG == 2 * RB_LT, "two digit groups per thread");

/* One block per (segment, range bucket): runs and partial sums of its c
   keys, which hold positions [O, O + c) of the segment's order. A thread
   holds at most RB_CAP / RB_LT keys, each |A * B| and A^2 at most n^2, so
   per-thread and block sums fit 64 bits for the n this path takes. */
__global__ void __launch_bounds__(RB_LT, 2) rb_local(int n, int m, int cap, int gmax,
                                                     const int *nspl, const unsigned *rcur,
                                                     const unsigned *boff, const u64 *bkey,
                                                     const int *bval, __int128 *part, int *ovf)
{
    extern __shared__ __align__(16) unsigned char sm[];
    u64 *sk = reinterpret_cast<u64 *>(sm);
    int *sv = reinterpret_cast<int *>(sk + RB_CAP);
    unsigned *gst = reinterpret_cast<unsigned *>(sv + RB_CAP);
    unsigned *cur = gst + RB_DIG + 1;
    unsigned char *mixed = reinterpret_cast<unsigned char *>(cur + RB_DIG);
    __shared__ u64 s_lo[RB_LT / 32], s_hi[RB_LT / 32];
    __shared__ unsigned wsum[RB_LT / 32];
    __shared__ long long ws[RB_LT / 32];
    __shared__ int s_skip;
    const int ls = blockIdx.x / m, idx = blockIdx.x % m;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    /* other blocks of the segment may raise its flag meanwhile: one read,
       shared, so the whole block takes the same branch */
    if (tid == 0) s_skip = *(volatile const int *)(ovf + ls) || idx > nspl[ls];
    for (int d = tid; d < RB_DIG; d += RB_LT) {
        cur[d] = 0u;
        mixed[d] = 0;
    }
    __syncthreads();
    if (s_skip) return;
    const int c = (int)rcur[(size_t)ls * RB_MAXB + idx];
    if (c > cap) return; /* the scan has flagged the segment */
    const long long O = boff[(size_t)ls * 2 * RB_MAXB + 2 * idx];
    const size_t base = ((size_t)ls * m + idx) * RB_CAP;
    const u64 *bk = bkey + base;
    const int *bv = bval + base;
    __int128 *pp = part + ((size_t)ls * 2 * RB_MAXB + 2 * idx) * 2;

    u64 lo = ~0ULL, hi = 0ULL;
    for (int q = tid; q < c; q += RB_LT) {
        const u64 k = bk[q];
        lo = k < lo ? k : lo;
        hi = k > hi ? k : hi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const u64 a = __shfl_xor_sync(0xffffffffu, lo, o), b = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if (lane == 0) {
        s_lo[w] = lo;
        s_hi[w] = hi;
    }
    __syncthreads();
    for (int k = 0; k < RB_LT / 32; ++k) {
        lo = s_lo[k] < lo ? s_lo[k] : lo;
        hi = s_hi[k] > hi ? s_hi[k] : hi;
    }
    if (c == 0 || lo == hi) {
        /* one run [O, O + c) */
        long long sb = 0;
        for (int q = tid; q < c; q += RB_LT) sb += bv[q];
        sb = rb_block_sum64<RB_LT>(sb, ws);
        if (tid == 0) {
            const long long A = 2 * O + c - n;
            pp[0] = (__int128)A * sb;
            pp[1] = (__int128)c * A * A;
        }
        return;
    }
    const int nbits = 64 - __clzll((long long)(hi - lo));
    const int shift = nbits > 10 ? nbits - 10 : 0;
    for (int q = tid; q < c; q += RB_LT) atomicAdd(&cur[(unsigned)((bk[q] - lo) >> shift)], 1u);
    __syncthreads();
    {
        const unsigned a0 = cur[2 * tid], a1 = cur[2 * tid + 1], t = a0 + a1;
        unsigned x = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        unsigned run = x - t;
        for (int k = 0; k < w; ++k) run += wsum[k];
        gst[2 * tid] = run;
        cur[2 * tid] = run;
        gst[2 * tid + 1] = run + a0;
        cur[2 * tid + 1] = run + a0;
        if (tid == 0) gst[RB_DIG] = (unsigned)c;
    }
    __syncthreads();
    for (int q = tid; q < c; q += RB_LT) {
        const u64 k = bk[q];
        const unsigned p = atomicAdd(&cur[(unsigned)((k - lo) >> shift)], 1u);
        sk[p] = k;
        sv[p] = bv[q];
    }
    __syncthreads();
    for (int q = tid; q < c; q += RB_LT) {
        const u64 k = sk[q];
        const unsigned d = (unsigned)((k - lo) >> shift);
        if (k != sk[gst[d]]) mixed[d] = 1;
    }
    __syncthreads();
    long long ab = 0, aa = 0;
    bool big = false;
    for (int q = tid; q < c; q += RB_LT) {
        const u64 k = sk[q];
        const unsigned d = (unsigned)((k - lo) >> shift);
        const unsigned gs = gst[d], ge = gst[d + 1];
        long long i = gs, j = ge;
        if (mixed[d]) {
            if (ge - gs <= (unsigned)gmax) {
                unsigned lt = 0, le = 0;
                for (unsigned t = gs; t < ge; ++t) {
                    const u64 o = sk[t];
                    lt += o < k;
                    le += o <= k;
                }
                i = gs + lt;
                j = gs + le;
            } else {
                big = true;
            }
        }
        const long long A = 2 * O + i + j - n;
        ab += A * (long long)sv[q];
        aa += A * A;
    }
    if (__syncthreads_or(big)) {
        /* the digit could not tell a large group apart (keys spread over many
           binades, as in a tail bucket): sort the bucket (bitonic, padded to
           a power of two by entries that order after every key, B marked
           INT_MIN) and take each key's run by binary search */
        int P2 = 1;
        while (P2 < c) P2 <<= 1;
        for (int q = c + tid; q < P2; q += RB_LT) {
            sk[q] = ~0ULL;
            sv[q] = INT_MIN;
        }
        __syncthreads();
        for (int k = 2; k <= P2; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = tid; i < P2; i += RB_LT) {
                    const int l = i ^ j;
                    if (l > i) {
                        const u64 a = sk[i], b = sk[l];
                        const int va = sv[i], vb = sv[l];
                        const bool agt = a > b || (a == b && va == INT_MIN && vb != INT_MIN);
                        if (agt == ((i & k) == 0)) {
                            sk[i] = b;
                            sk[l] = a;
                            sv[i] = vb;
                            sv[l] = va;
                        }
                    }
                }
                __syncthreads();
            }
        ab = 0;
        aa = 0;
        for (int q = tid; q < c; q += RB_LT) {
            const u64 k = sk[q];
            const long long A = 2 * O + rk_lower(sk, 0, c, k) + rk_upper(sk, 0, c, k) - n;
            ab += A * (long long)sv[q];
            aa += A * A;
        }
    }
    const long long sab = rb_block_sum64<RB_LT>(ab, ws);
    const long long saa = rb_block_sum64<RB_LT>(aa, ws);
    if (tid == 0) {
        pp[0] = sab;
        pp[1] = saa;
    }
}

/* One block per segment not flagged: the bucket partials summed into the
   two 128-bit sums, written as rk_final writes them. */
__global__ void __launch_bounds__(RS_T) rb_final(const int *nspl, const __int128 *part,
                                                 const int *ovf, u64 *out)
{
    __shared__ __int128 red[RS_T];
    const int ls = blockIdx.x, tid = threadIdx.x;
    if (ovf[ls]) return;
    const int nb = 2 * nspl[ls] + 1;
    __int128 ab = 0, aa = 0;
    for (int b = tid; b < nb; b += RS_T) {
        const size_t e = (size_t)ls * 2 * RB_MAXB + b;
        ab += part[e * 2 + 0];
        aa += part[e * 2 + 1];
    }
    const unsigned __int128 uab = (unsigned __int128)rk_block_sum(ab, red);
    const unsigned __int128 uaa = (unsigned __int128)rk_block_sum(aa, red);
    if (tid == 0) {
        out[(size_t)ls * 4 + 0] = (u64)(uab >> 64);
        out[(size_t)ls * 4 + 1] = (u64)uab;
        out[(size_t)ls * 4 + 2] = (u64)(uaa >> 64);
        out[(size_t)ls * 4 + 3] = (u64)uaa;
    }
}

/* ---- order statistics --------------------------------------------------- */

#define OS_T 256

/* Median (what 0) or interquartile mean (what 1) of a sorted segment of
   |r| patterns (eval.cu:4436-4520 semantics): the middle value or the mean of
   the two middle values; the mean of ranks [n/4, 3n/4) (all rows below four)
   as a fixed 256-thread strided sum and tree. */
__global__ void __launch_bounds__(OS_T) os_pick(const u64 *ka, const u64 *kb,
                                                const unsigned char *par, int n, int seg0,
                                                int nseg, int what, const int *status,
                                                double *out)
{
    __shared__ double part[OS_T];
    const int ls = blockIdx.x;
    const int seg = seg0 + ls;
    const int tid = threadIdx.x;
    if (ls >= nseg) return;
    if (status[seg] != 0) {
        if (tid == 0) out[seg] = CUDART_NAN;
        return;
    }
    const u64 *k = (par[ls] ? kb : ka) + (size_t)ls * n;
    if (what == 0) {
        if (tid == 0)
            out[seg] = (n & 1) ? rk_key_abs_value(k[n / 2])
                               : 0.5 * (rk_key_abs_value(k[n / 2 - 1]) + rk_key_abs_value(k[n / 2]));
        return;
    }
    const int lo = n < 4 ? 0 : n / 4, hi = n < 4 ? n : (3 * n) / 4;
    double s = 0.0;
    for (int i = lo + tid; i < hi; i += OS_T) s += rk_key_abs_value(k[i]);
    part[tid] = s;
    __syncthreads();
    for (int st = OS_T / 2; st > 0; st >>= 1) {
        if (tid < st) part[tid] += part[tid + st];
        __syncthreads();
    }
    if (tid == 0) out[seg] = part[0] / (double)(hi - lo);
}

/* ---- maximum-error scan ------------------------------------------------- */

#define MX_T 256

/* One block per segment (eval.cu:4522-4640 semantics): rows tid, tid + 256,
   ...; the integer max of the |r| patterns with the lowest attaining row;
   with a coordinate and a finite level t, the intersection of the per-row
   intervals {delta : |r + b delta| <= t}, b = dr/dc from the reverse sweep,
   where a row with b = 0 only vetoes (|r| > t). A row that is not finite
   stops the thread and marks the segment. */
__global__ void __launch_bounds__(MX_T) mx_scan(const FIns *fins, const int *fins_off,
                                                const int4 *finfo, const int *valid,
                                                const int *pcount, const double *c0, int kmax,
                                                const int *coords, const double *levels,
                                                const double *cols, const double *y, int npad,
                                                int n, int ntrials, int maxins, RcMaxOut *out)
{
    using V4 = FiV<double, 1>::V4;
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ u64 skey[MX_T];
    __shared__ int srow[MX_T];
    __shared__ double slo[MX_T], shi[MX_T];
    __shared__ int sbad[MX_T];
    const int seg = blockIdx.x;
    const int tid = threadIdx.x;
    const int cand = seg / ntrials;
    const int4 info = finfo[cand];
    const int nf = info.x, nr = info.y, slots = info.w & 0xffff, ntape = info.w >> 16;
    const int p = pcount[cand];
    FIns *ins = reinterpret_cast<FIns *>(sm);
    double *cv = reinterpret_cast<double *>(sm + 8 * (size_t)((maxins + 1) & ~1));
    V4 *stk = reinterpret_cast<V4 *>(cv + FT_MAX_CONST);
    V4 *tape = stk + (size_t)slots * MX_T;
    double *g = reinterpret_cast<double *>(tape + (size_t)ntape * MX_T);
    const bool ok = valid[cand] != 0;
    if (ok) {
        for (int i = tid; i < nf + nr; i += MX_T) ins[i] = fins[fins_off[cand] + i];
        if (tid < FT_MAX_CONST) cv[tid] = tid < kmax ? c0[(size_t)seg * kmax + tid] : 0.0;
    }
    __syncthreads();
    const int coord = (coords && p > 0 && coords[seg] >= 0 && coords[seg] < p) ? coords[seg] : -1;
    const double level = levels ? levels[seg] : CUDART_NAN;
    const bool want = coord >= 0 && isfinite(level) && level >= 0.0;
    u64 mykey = 0ULL;
    int myrow = 0x7fffffff;
    double mylo = -CUDART_INF, myhi = CUDART_INF;
    int mybad = ok ? 0 : 1;
    for (int row = tid; ok && row < n; row += MX_T) {
        double pr;
        if (want) fi_forward<double, 1, true>(ins, cv, cols, npad, row, stk, tape, MX_T, tid, &pr);
        else fi_forward<double, 1, false>(ins, cv, cols, npad, row, stk, nullptr, MX_T, tid, &pr);
        const double r = pr - y[row];
        if (!isfinite(pr) || fabs(pr) > 1e30 || !isfinite(r)) {
            mybad |= 1;
            break;
        }
        const u64 key = rk_abs_key(r);
        if (key > mykey || (key == mykey && row < myrow)) {
            mykey = key;
            myrow = row;
        }
        if (want && (mybad & 2) == 0) {
            for (int j = 0; j < p; ++j) g[(size_t)j * MX_T + tid] = 0.0;
            double seed = 1.0;
            fi_reverse<double, 1>(ins + nf, nr, stk, tape, MX_T, tid, g + tid, MX_T, MX_T, &seed);
            const double b = g[(size_t)coord * MX_T + tid];
            if (!isfinite(b)) {
                mybad |= 1;
                break;
            }
            if (b == 0.0) {
                if (fabs(r) > level) mybad |= 2;
            } else {
                const double e1 = (-level - r) / b;
                const double e2 = (level - r) / b;
                mylo = fmax(mylo, fmin(e1, e2));
                myhi = fmin(myhi, fmax(e1, e2));
            }
        }
    }
    skey[tid] = mykey;
    srow[tid] = myrow;
    slo[tid] = mylo;
    shi[tid] = myhi;
    sbad[tid] = mybad;
    __syncthreads();
    for (int st = MX_T / 2; st > 0; st >>= 1) {
        if (tid < st) {
            const int j = tid + st;
            if (skey[j] > skey[tid] || (skey[j] == skey[tid] && srow[j] < srow[tid])) {
                skey[tid] = skey[j];
                srow[tid] = srow[j];
            }
            slo[tid] = fmax(slo[tid], slo[j]);
            shi[tid] = fmin(shi[tid], shi[j]);
            sbad[tid] |= sbad[j];
        }
        __syncthreads();
    }
    if (tid == 0) {
        const int bad = sbad[0];
        RcMaxOut o;
        o.status = (bad & 1) ? 2 : 0;
        o.vmax = (bad & 1) ? CUDART_NAN : rk_key_abs_value(skey[0]);
        o.row = (bad & 1) ? -1 : srow[0];
        o.lo = (bad & 2) ? CUDART_INF : slo[0];
        o.hi = (bad & 2) ? -CUDART_INF : shi[0];
        out[seg] = o;
    }
}

/* ---- host side -------------------------------------------------------- */

namespace {

size_t rs_bytes(size_t keys, int nseg, int n, bool vals)
{
    const size_t ntiles = (size_t)((n + RS_TILE - 1) / RS_TILE);
    size_t s = 2 * sizeof(u64) * keys + (vals ? 2 * sizeof(unsigned int) * keys : 0);
    s += sizeof(unsigned int) * RS_PASSES * 256 * (size_t)nseg;
    s += sizeof(u64) * 256 * ntiles * (size_t)nseg;
    s += 2 * (size_t)nseg + sizeof(int) * RS_PASSES + 8 * 256;
    s += 2 * sizeof(__int128) * ntiles * (size_t)nseg;
    return s;
}

/* Carve the sort buffers for `nseg` segments of n keys from `base` at *cur. */
RsBuffers rs_carve(unsigned char *base, size_t *cur, int nseg, int n, bool vals, __int128 **part)
{
    const size_t keys = (size_t)nseg * n;
    const size_t ntiles = (size_t)((n + RS_TILE - 1) / RS_TILE);
    RsBuffers b;
    b.ka = reinterpret_cast<u64 *>(base + rc_take(cur, sizeof(u64) * keys));
    b.kb = reinterpret_cast<u64 *>(base + rc_take(cur, sizeof(u64) * keys));
    b.va = vals ? reinterpret_cast<unsigned int *>(base + rc_take(cur, sizeof(unsigned int) * keys))
                : nullptr;
    b.vb = vals ? reinterpret_cast<unsigned int *>(base + rc_take(cur, sizeof(unsigned int) * keys))
                : nullptr;
    b.count = reinterpret_cast<unsigned int *>(
        base + rc_take(cur, sizeof(unsigned int) * RS_PASSES * 256 * (size_t)nseg));
    b.state = reinterpret_cast<u64 *>(base + rc_take(cur, sizeof(u64) * 256 * ntiles * (size_t)nseg));
    b.ticket = reinterpret_cast<int *>(base + rc_take(cur, sizeof(int) * RS_PASSES));
    b.par = base + rc_take(cur, (size_t)nseg);
    b.skip = base + rc_take(cur, (size_t)nseg);
    *part = reinterpret_cast<__int128 *>(base + rc_take(cur, 2 * sizeof(__int128) * ntiles * nseg));
    return b;
}

/* B (the target's doubled centred ranks) and sum B^2, once per context. */
int rk_prepare(RcCtx *c)
{
    if (c->rank_ready) return 0;
    if (c->n <= 1) return -1;
    if (rc_ensure_f64(c) != 0) return -1;
    const int n = c->n;
    if (!c->d_rank_b && cudaMalloc((void **)&c->d_rank_b, sizeof(long long) * (size_t)n) != cudaSuccess) {
        cudaGetLastError();
        c->d_rank_b = nullptr;
        return -1;
    }
    size_t cur = 0;
    const size_t o_out = rc_take(&cur, sizeof(u64) * 4);
    const size_t o_abort = rc_take(&cur, sizeof(int));
    const size_t io_end = rc_take(&cur, 0);
    const size_t work = cur;
    if (rc_reserve(c, work + rs_bytes((size_t)n, 1, n, true) + 4096, io_end) != 0) return -1;
    int *d_abort = reinterpret_cast<int *>(c->dev + o_abort);
    cudaMemsetAsync(d_abort, 0, sizeof(int), c->s);
    __int128 *part = nullptr;
    size_t wc = work;
    const RsBuffers b = rs_carve(c->dev, &wc, 1, n, true, &part);
    const int ntiles = (n + RS_TILE - 1) / RS_TILE;
    rk_target_keys<<<(n + 255) / 256, 256, 0, c->s>>>(c->d_y64, n, b.ka, b.va);
    c->launches += 3 + rs_sort<true>(b, 1, n, d_abort, c->s, false);
    rk_runs<RK_FILL><<<ntiles, RS_T, 0, c->s>>>(b.ka, b.kb, b.va, b.vb, b.par, n, ntiles, nullptr,
                                                c->d_rank_b, part);
    rk_final<<<1, RS_T, 0, c->s>>>(part, ntiles, reinterpret_cast<u64 *>(c->dev + o_out));
    cudaMemcpyAsync(c->host + o_out, c->dev + o_out, io_end - o_out, cudaMemcpyDeviceToHost, c->s);
    if (rc_finish(c) != 0) return -1;
    if (*reinterpret_cast<const int *>(c->host + o_abort) != 0) return -1;
    /* sum A^2 of the target is sum B^2 */
    const u64 *h = reinterpret_cast<const u64 *>(c->host + o_out);
    c->rank_bb[0] = h[2];
    c->rank_bb[1] = h[3];
    c->rank_ready = 1;
    return 0;
}

struct StatPrep {
    FitPrep b;
    size_t o_fins, o_finsoff, o_finfo, o_valid, o_p, o_c0, in_end;
};

/* Upload the decoded programs and the per-segment constants. */
void stat_inputs(RcCtx *c, const unsigned int *prog, const unsigned int *off, const int *pcount,
                 int nsets, int nsegs, int kmax, const double *c0, size_t *cur, StatPrep &sp)
{
    prep_batch(off, prog, pcount, nsets, c->v, sp.b);
    sp.o_fins = rc_take(cur, sizeof(FIns) * sp.b.fins.size());
    sp.o_finsoff = rc_take(cur, sizeof(int) * (nsets + 1));
    sp.o_finfo = rc_take(cur, sizeof(int4) * nsets);
    sp.o_valid = rc_take(cur, sizeof(int) * nsets);
    sp.o_p = rc_take(cur, sizeof(int) * nsets);
    sp.o_c0 = rc_take(cur, sizeof(double) * (size_t)nsegs * kmax);
    sp.in_end = rc_take(cur, 0);
}

void stat_copy(RcCtx *c, const int *pcount, int nsets, int nsegs, int kmax, const double *c0,
               const StatPrep &sp)
{
    unsigned char *h = c->host;
    memcpy(h + sp.o_fins, sp.b.fins.data(), sizeof(FIns) * sp.b.fins.size());
    memcpy(h + sp.o_finsoff, sp.b.fins_off.data(), sizeof(int) * (nsets + 1));
    memcpy(h + sp.o_finfo, sp.b.finfo.data(), sizeof(int4) * nsets);
    memcpy(h + sp.o_valid, sp.b.valid.data(), sizeof(int) * nsets);
    memcpy(h + sp.o_p, pcount, sizeof(int) * nsets);
    memcpy(h + sp.o_c0, c0, sizeof(double) * (size_t)nsegs * kmax);
    cudaMemcpyAsync(c->dev, h, sp.in_end, cudaMemcpyHostToDevice, c->s);
}

size_t key_smem(const StatPrep &sp)
{
    return 8 * (size_t)((sp.b.fmaxins + 1) & ~1) + 8 * FT_MAX_CONST +
           16 * (size_t)(sp.b.fslots > 0 ? sp.b.fslots : 1) * RK_T;
}

/* Segments per wave so that a wave's sort buffers stay within the budget. */
int wave_segments(int nsegs, int n, bool vals)
{
    const size_t per = rs_bytes((size_t)n, 1, n, vals);
    size_t w = RK_WAVE_BYTES / (per ? per : 1);
    if (w < 1) w = 1;
    return (int)std::min<size_t>(w, (size_t)nsegs);
}

/* Range buckets of the bucketed sums for n rows: one up to RB_CAP rows,
   else ceil(n / RB_AVG); 0 past the rows the path takes (RB_AVG * RB_MAXB). */
int rb_buckets(int n)
{
    if (n <= RB_CAP) return 1;
    const long long m = ((long long)n + RB_AVG - 1) / RB_AVG;
    return m <= RB_MAXB ? (int)m : 0;
}

struct RbBuffers {
    u64 *keys;                /* [nseg][n] keys in row order */
    u64 *samp;                /* [nseg][RB_MAXS] sample keys */
    u64 *spl;                 /* [nseg][RB_MAXB] splitters */
    int *nspl;                /* [nseg] */
    u64 *bkey;                /* [nseg][m][RB_CAP] range-bucket slots */
    int *bval;                /* [nseg][m][RB_CAP] their B */
    unsigned *rcur, *ecnt;    /* [nseg][RB_MAXB] range / equality bucket sizes */
    unsigned long long *esum; /* [nseg][RB_MAXB] equality buckets' B sums */
    unsigned *boff;           /* [nseg][2 * RB_MAXB] first positions */
    __int128 *part;           /* [nseg][2 * RB_MAXB][2] bucket partial sums */
    unsigned char *zero;      /* rcur, ecnt and esum, zeroed per wave */
    size_t zero_bytes;
};

size_t rb_bytes(int nseg, int n, int m)
{
    const size_t ns = (size_t)nseg;
    size_t s = sizeof(u64) * ns * (size_t)n + sizeof(u64) * ns * (RB_MAXS + RB_MAXB) +
               sizeof(int) * ns;
    s += (sizeof(u64) + sizeof(int)) * ns * (size_t)m * RB_CAP;
    s += (2 * sizeof(unsigned) + sizeof(unsigned long long)) * ns * RB_MAXB;
    s += sizeof(unsigned) * ns * 2 * RB_MAXB + 2 * sizeof(__int128) * ns * 2 * RB_MAXB;
    return s + 16 * 256;
}

RbBuffers rb_carve(unsigned char *base, size_t *cur, int nseg, int n, int m)
{
    const size_t ns = (size_t)nseg;
    RbBuffers r;
    r.keys = reinterpret_cast<u64 *>(base + rc_take(cur, sizeof(u64) * ns * (size_t)n));
    r.samp = reinterpret_cast<u64 *>(base + rc_take(cur, sizeof(u64) * ns * RB_MAXS));
    r.spl = reinterpret_cast<u64 *>(base + rc_take(cur, sizeof(u64) * ns * RB_MAXB));
    r.nspl = reinterpret_cast<int *>(base + rc_take(cur, sizeof(int) * ns));
    r.bkey = reinterpret_cast<u64 *>(base + rc_take(cur, sizeof(u64) * ns * (size_t)m * RB_CAP));
    r.bval = reinterpret_cast<int *>(base + rc_take(cur, sizeof(int) * ns * (size_t)m * RB_CAP));
    r.zero_bytes = (2 * sizeof(unsigned) + sizeof(unsigned long long)) * ns * RB_MAXB;
    r.zero = base + rc_take(cur, r.zero_bytes);
    r.rcur = reinterpret_cast<unsigned *>(r.zero);
    r.ecnt = r.rcur + ns * RB_MAXB;
    r.esum = reinterpret_cast<unsigned long long *>(r.ecnt + ns * RB_MAXB);
    r.boff = reinterpret_cast<unsigned *>(base + rc_take(cur, sizeof(unsigned) * ns * 2 * RB_MAXB));
    r.part = reinterpret_cast<__int128 *>(
        base + rc_take(cur, 2 * sizeof(__int128) * ns * 2 * RB_MAXB));
    return r;
}

#define RB_WAVE_BYTES ((size_t)4 << 30)

int rb_wave_segments(int nsegs, int n, int m)
{
    const size_t per = rb_bytes(1, n, m);
    size_t w = RB_WAVE_BYTES / (per ? per : 1);
    if (w < 1) w = 1;
    return (int)std::min<size_t>(w, (size_t)nsegs);
}

}  // namespace

extern "C" {

float rc_rank_score_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                          const int *pcount, int nsets, int ntrials, int kmax, const double *c0,
                          unsigned long long *out, int *out_status, unsigned long long *out_bb)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !prog || !off || !pcount || !c0 || !out || !out_status || !out_bb) return -1.0f;
    if (nsets <= 0 || ntrials <= 0 || kmax <= 0 || kmax > FT_MAX_CONST) return -1.0f;
    if (c->n <= 1) return -1.0f;
    const int n = c->n;
    const long long total = (long long)nsets * ntrials * (long long)n;
    if (total > 0x7fffffffLL) return -1.0f;
    if (rk_prepare(c) != 0) return -1.0f;
    const int nsegs = nsets * ntrials;
    /* the bucketed sums unless turned off or past their rows */
    const int m = c->rank_cap < 0 ? 0 : rb_buckets(n);
    const int cap = c->rank_cap > 0 ? std::min(c->rank_cap, RB_CAP) : RB_CAP;
    const int gmax = c->rank_gmax > 0 ? c->rank_gmax : RB_GMAX;
    StatPrep sp;
    size_t cur = 0;
    stat_inputs(c, prog, off, pcount, nsets, nsegs, kmax, c0, &cur, sp);
    const size_t o_out = rc_take(&cur, sizeof(u64) * 4 * (size_t)nsegs);
    const size_t o_status = rc_take(&cur, sizeof(int) * (size_t)nsegs);
    const size_t o_ovf = rc_take(&cur, sizeof(int) * (size_t)nsegs);
    const size_t o_abort = rc_take(&cur, sizeof(int));
    const size_t io_end = rc_take(&cur, 0);
    const int wseg = m > 0 ? rb_wave_segments(nsegs, n, m) : wave_segments(nsegs, n, true);
    const size_t work = cur;
    const size_t wbytes = m > 0 ? std::max(rb_bytes(wseg, n, m), rs_bytes((size_t)n, 1, n, true))
                                : rs_bytes((size_t)wseg * n, wseg, n, true);
    if (rc_reserve(c, work + wbytes + 4096, io_end) != 0) return -1.0f;
    stat_copy(c, pcount, nsets, nsegs, kmax, c0, sp);
    unsigned char *dev = c->dev;
    int *d_status = reinterpret_cast<int *>(dev + o_status);
    int *d_ovf = reinterpret_cast<int *>(dev + o_ovf);
    int *d_abort = reinterpret_cast<int *>(dev + o_abort);
    u64 *d_out = reinterpret_cast<u64 *>(dev + o_out);
    cudaMemsetAsync(d_status, 0, sizeof(int) * nsegs, c->s);
    cudaMemsetAsync(d_ovf, 0, sizeof(int) * nsegs, c->s);
    cudaMemsetAsync(d_abort, 0, sizeof(int), c->s);
    const size_t smem = key_smem(sp);
    if (rc_raise_smem((const void *)rk_keys<RK_RANK>, smem) != 0) return -1.0f;
    if (m > 0 && (rc_raise_smem((const void *)rb_sample, smem) != 0 ||
                  rc_raise_smem((const void *)rb_splitters, sizeof(u64) * RB_MAXS) != 0 ||
                  rc_raise_smem((const void *)rb_local, rb_local_smem()) != 0))
        return -1.0f;
    const int ktiles = (n + RK_TILE - 1) / RK_TILE;
    const int ntiles = (n + RS_TILE - 1) / RS_TILE;
    const FIns *d_fins = reinterpret_cast<const FIns *>(dev + sp.o_fins);
    const int *d_finsoff = reinterpret_cast<const int *>(dev + sp.o_finsoff);
    const int4 *d_finfo = reinterpret_cast<const int4 *>(dev + sp.o_finfo);
    const int *d_valid = reinterpret_cast<const int *>(dev + sp.o_valid);
    const double *d_c0 = reinterpret_cast<const double *>(dev + sp.o_c0);
    /* the radix-sort sums of segments [s0, s0 + ns) */
    auto radix_wave = [&](int s0, int ns) {
        size_t wc = work;
        __int128 *part = nullptr;
        const RsBuffers b = rs_carve(dev, &wc, ns, n, true, &part);
        cudaMemsetAsync(b.count, 0, sizeof(unsigned int) * RS_PASSES * 256 * (size_t)ns, c->s);
        rk_keys<RK_RANK><<<(unsigned)ns * ktiles, RK_T, smem, c->s>>>(
            d_fins, d_finsoff, d_finfo, d_valid, d_c0, kmax, c->d_cols64, c->d_y64, c->npad, n,
            ntrials, s0, ktiles, sp.b.fmaxins, b.ka, b.va, b.count, d_status);
        c->launches += 3 + rs_sort<true>(b, ns, n, d_abort, c->s, true);
        rk_runs<RK_SUMS><<<(unsigned)ns * ntiles, RS_T, 0, c->s>>>(
            b.ka, b.kb, b.va, b.vb, b.par, n, ntiles, c->d_rank_b, nullptr, part);
        rk_final<<<ns, RS_T, 0, c->s>>>(part, ntiles, d_out + 4 * (size_t)s0);
    };
    /* the bucketed sums of segments [s0, s0 + ns); a flagged segment is left
       to the radix sort */
    auto bucket_wave = [&](int s0, int ns) {
        size_t wc = work;
        const RbBuffers r = rb_carve(dev, &wc, ns, n, m);
        cudaMemsetAsync(r.zero, 0, r.zero_bytes, c->s);
        if (m > 1) {
            const int S = RB_OVS * m;
            int P2 = 1;
            while (P2 < S) P2 <<= 1;
            const int sblocks = (S / 2 + RK_T - 1) / RK_T;
            rb_sample<<<(unsigned)ns * sblocks, RK_T, smem, c->s>>>(
                d_fins, d_finsoff, d_finfo, d_valid, d_c0, kmax, c->d_cols64, c->npad, n, ntrials,
                s0, sblocks, S, sp.b.fmaxins, r.samp);
            rb_splitters<<<ns, RB_ST, sizeof(u64) * P2, c->s>>>(r.samp, S, P2, m, r.spl, r.nspl);
            c->launches += 2;
        } else {
            cudaMemsetAsync(r.nspl, 0, sizeof(int) * ns, c->s);
        }
        rk_keys<RK_RANK><<<(unsigned)ns * ktiles, RK_T, smem, c->s>>>(
            d_fins, d_finsoff, d_finfo, d_valid, d_c0, kmax, c->d_cols64, c->d_y64, c->npad, n,
            ntrials, s0, ktiles, sp.b.fmaxins, r.keys, nullptr, nullptr, d_status);
        const int ctiles = (n + RB_CT - 1) / RB_CT;
        rb_scatter<<<(unsigned)ns * ctiles, RB_CTT, 0, c->s>>>(
            r.keys, n, ctiles, m, cap, c->d_rank_b, r.spl, r.nspl, r.rcur, r.ecnt, r.esum, r.bkey,
            r.bval, d_ovf + s0);
        rb_scan<<<ns, RB_ST, 0, c->s>>>(n, cap, r.nspl, r.rcur, r.ecnt, r.esum, r.boff, r.part,
                                        d_ovf + s0);
        rb_local<<<(unsigned)ns * m, RB_LT, rb_local_smem(), c->s>>>(
            n, m, cap, gmax, r.nspl, r.rcur, r.boff, r.bkey, r.bval, r.part, d_ovf + s0);
        rb_final<<<ns, RS_T, 0, c->s>>>(r.nspl, r.part, d_ovf + s0, d_out + 4 * (size_t)s0);
        c->launches += 5;
    };
    cudaEventRecord(c->t0, c->s);
    for (int s0 = 0; s0 < nsegs; s0 += wseg) {
        const int ns = std::min(wseg, nsegs - s0);
        if (m > 0) bucket_wave(s0, ns);
        else radix_wave(s0, ns);
    }
    cudaEventRecord(c->t1, c->s);
    if (cudaGetLastError() != cudaSuccess) return -1.0f;
    cudaMemcpyAsync(c->host + sp.in_end, dev + sp.in_end, io_end - sp.in_end,
                    cudaMemcpyDeviceToHost, c->s);
    if (rc_finish(c) != 0) return -1.0f;
    if (*reinterpret_cast<const int *>(c->host + o_abort) != 0) return -1.0f;
    c->rank_fallbacks = m > 0 ? 0 : nsegs;
    if (m > 0) {
        /* segments the buckets could not take: the radix sort, one each */
        const int *h_ovf = reinterpret_cast<const int *>(c->host + o_ovf);
        std::vector<int> redo;
        for (int s = 0; s < nsegs; ++s)
            if (h_ovf[s]) redo.push_back(s);
        if (!redo.empty()) {
            for (int s : redo) radix_wave(s, 1);
            cudaEventRecord(c->t1, c->s);
            if (cudaGetLastError() != cudaSuccess) return -1.0f;
            cudaMemcpyAsync(c->host + sp.in_end, dev + sp.in_end, io_end - sp.in_end,
                            cudaMemcpyDeviceToHost, c->s);
            if (rc_finish(c) != 0) return -1.0f;
            if (*reinterpret_cast<const int *>(c->host + o_abort) != 0) return -1.0f;
        }
        c->rank_fallbacks = (int)redo.size();
    }
    memcpy(out, c->host + o_out, sizeof(u64) * 4 * (size_t)nsegs);
    memcpy(out_status, c->host + o_status, sizeof(int) * (size_t)nsegs);
    out_bb[0] = c->rank_bb[0];
    out_bb[1] = c->rank_bb[1];
    float ms = -1.0f;
    cudaEventElapsedTime(&ms, c->t0, c->t1);
    return ms;
}

int rc_rank_tuning(void *ctx, int bucket_cap, int group_max)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || bucket_cap < -1 || bucket_cap > RB_CAP || group_max < 0) return -1;
    c->rank_cap = bucket_cap;
    c->rank_gmax = group_max;
    return 0;
}

int rc_rank_last_fallbacks(void *ctx)
{
    RcCtx *c = (RcCtx *)ctx;
    return c ? c->rank_fallbacks : -1;
}

int rc_rank_debug_b(void *ctx, long long *out)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !out) return -1;
    if (rk_prepare(c) != 0) return -1;
    if (cudaMemcpy(out, c->d_rank_b, sizeof(long long) * (size_t)c->n, cudaMemcpyDeviceToHost) !=
        cudaSuccess)
        return -1;
    return 0;
}

float rc_order_stat_score_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                                const int *pcount, int nsets, int ntrials, int kmax,
                                const double *c0, int what, double *out_value, int *out_status)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !prog || !off || !pcount || !c0 || !out_value || !out_status) return -1.0f;
    if (nsets <= 0 || ntrials <= 0 || kmax <= 0 || kmax > FT_MAX_CONST) return -1.0f;
    if (what != 0 && what != 1) return -1.0f;
    if (c->n <= 0) return -1.0f;
    const int n = c->n;
    const long long total = (long long)nsets * ntrials * (long long)n;
    if (total > 0x7fffffffLL) return -1.0f;
    if (rc_ensure_f64(c) != 0) return -1.0f;
    const int nsegs = nsets * ntrials;
    StatPrep sp;
    size_t cur = 0;
    stat_inputs(c, prog, off, pcount, nsets, nsegs, kmax, c0, &cur, sp);
    const size_t o_val = rc_take(&cur, sizeof(double) * (size_t)nsegs);
    const size_t o_status = rc_take(&cur, sizeof(int) * (size_t)nsegs);
    const size_t o_abort = rc_take(&cur, sizeof(int));
    const size_t io_end = rc_take(&cur, 0);
    const int wseg = wave_segments(nsegs, n, false);
    const size_t work = cur;
    if (rc_reserve(c, work + rs_bytes((size_t)wseg * n, wseg, n, false) + 4096, io_end) != 0)
        return -1.0f;
    stat_copy(c, pcount, nsets, nsegs, kmax, c0, sp);
    unsigned char *dev = c->dev;
    int *d_status = reinterpret_cast<int *>(dev + o_status);
    int *d_abort = reinterpret_cast<int *>(dev + o_abort);
    cudaMemsetAsync(d_status, 0, sizeof(int) * nsegs, c->s);
    cudaMemsetAsync(d_abort, 0, sizeof(int), c->s);
    const size_t smem = key_smem(sp);
    if (rc_raise_smem((const void *)rk_keys<RK_ABS>, smem) != 0) return -1.0f;
    const int ktiles = (n + RK_TILE - 1) / RK_TILE;
    cudaEventRecord(c->t0, c->s);
    for (int s0 = 0; s0 < nsegs; s0 += wseg) {
        const int ns = std::min(wseg, nsegs - s0);
        size_t wc = work;
        __int128 *part = nullptr;
        const RsBuffers b = rs_carve(dev, &wc, ns, n, false, &part);
        cudaMemsetAsync(b.count, 0, sizeof(unsigned int) * RS_PASSES * 256 * (size_t)ns, c->s);
        rk_keys<RK_ABS><<<(unsigned)ns * ktiles, RK_T, smem, c->s>>>(
            reinterpret_cast<const FIns *>(dev + sp.o_fins),
            reinterpret_cast<const int *>(dev + sp.o_finsoff),
            reinterpret_cast<const int4 *>(dev + sp.o_finfo),
            reinterpret_cast<const int *>(dev + sp.o_valid),
            reinterpret_cast<const double *>(dev + sp.o_c0), kmax, c->d_cols64, c->d_y64, c->npad,
            n, ntrials, s0, ktiles, sp.b.fmaxins, b.ka, nullptr, b.count, d_status);
        c->launches += 2 + rs_sort<false>(b, ns, n, d_abort, c->s, true);
        os_pick<<<ns, OS_T, 0, c->s>>>(b.ka, b.kb, b.par, n, s0, ns, what, d_status,
                                       reinterpret_cast<double *>(dev + o_val));
    }
    cudaEventRecord(c->t1, c->s);
    if (cudaGetLastError() != cudaSuccess) return -1.0f;
    cudaMemcpyAsync(c->host + sp.in_end, dev + sp.in_end, io_end - sp.in_end,
                    cudaMemcpyDeviceToHost, c->s);
    if (rc_finish(c) != 0) return -1.0f;
    if (*reinterpret_cast<const int *>(c->host + o_abort) != 0) return -1.0f;
    memcpy(out_value, c->host + o_val, sizeof(double) * (size_t)nsegs);
    memcpy(out_status, c->host + o_status, sizeof(int) * (size_t)nsegs);
    float ms = -1.0f;
    cudaEventElapsedTime(&ms, c->t0, c->t1);
    return ms;
}

float rc_max_scan_batch(void *ctx, const unsigned int *prog, const unsigned int *off,
                        const int *pcount, int nsets, int ntrials, int kmax, const double *c0,
                        const int *coords, const double *levels, RcMaxOut *out)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !prog || !off || !pcount || !c0 || !out) return -1.0f;
    if (nsets <= 0 || ntrials <= 0 || kmax <= 0 || kmax > FT_MAX_CONST) return -1.0f;
    if (c->n <= 0) return -1.0f;
    const int n = c->n;
    const int nsegs = nsets * ntrials;
    if ((long long)nsegs * (long long)n > 0x7fffffffLL) return -1.0f;
    if (rc_ensure_f64(c) != 0) return -1.0f;
    StatPrep sp;
    size_t cur = 0;
    stat_inputs(c, prog, off, pcount, nsets, nsegs, kmax, c0, &cur, sp);
    const size_t o_coords = rc_take(&cur, sizeof(int) * (size_t)nsegs);
    const size_t o_levels = rc_take(&cur, sizeof(double) * (size_t)nsegs);
    const size_t in_end = rc_take(&cur, 0);
    const size_t o_out = rc_take(&cur, sizeof(RcMaxOut) * (size_t)nsegs);
    const size_t io_end = rc_take(&cur, 0);
    if (rc_reserve(c, io_end, io_end) != 0) return -1.0f;
    int *hc = reinterpret_cast<int *>(c->host + o_coords);
    double *hl = reinterpret_cast<double *>(c->host + o_levels);
    for (int s = 0; s < nsegs; ++s) {
        hc[s] = coords ? coords[s] : -1;
        hl[s] = (coords && levels) ? levels[s] : std::numeric_limits<double>::quiet_NaN();
    }
    stat_copy(c, pcount, nsets, nsegs, kmax, c0, sp);
    cudaMemcpyAsync(c->dev + o_coords, c->host + o_coords, in_end - o_coords,
                    cudaMemcpyHostToDevice, c->s);
    unsigned char *dev = c->dev;
    const int pmax = std::max(sp.b.pmax, 1);
    const size_t smem = 8 * (size_t)((sp.b.fmaxins + 1) & ~1) + 8 * FT_MAX_CONST +
                        8 * (size_t)MX_T * (sp.b.fslots + sp.b.ftape + pmax);
    if (smem > 200 * 1024) return -1.0f;
    if (rc_raise_smem((const void *)mx_scan, smem) != 0) return -1.0f;
    cudaEventRecord(c->t0, c->s);
    c->launches += 1;
    mx_scan<<<nsegs, MX_T, smem, c->s>>>(
        reinterpret_cast<const FIns *>(dev + sp.o_fins),
        reinterpret_cast<const int *>(dev + sp.o_finsoff),
        reinterpret_cast<const int4 *>(dev + sp.o_finfo),
        reinterpret_cast<const int *>(dev + sp.o_valid), reinterpret_cast<const int *>(dev + sp.o_p),
        reinterpret_cast<const double *>(dev + sp.o_c0), kmax,
        reinterpret_cast<const int *>(dev + o_coords), reinterpret_cast<const double *>(dev + o_levels),
        c->d_cols64, c->d_y64, c->npad, n, ntrials, sp.b.fmaxins,
        reinterpret_cast<RcMaxOut *>(dev + o_out));
    cudaEventRecord(c->t1, c->s);
    if (cudaGetLastError() != cudaSuccess) return -1.0f;
    cudaMemcpyAsync(c->host + o_out, dev + o_out, sizeof(RcMaxOut) * nsegs, cudaMemcpyDeviceToHost,
                    c->s);
    if (rc_finish(c) != 0) return -1.0f;
    memcpy(out, c->host + o_out, sizeof(RcMaxOut) * (size_t)nsegs);
    float ms = -1.0f;
    cudaEventElapsedTime(&ms, c->t0, c->t1);
    return ms;
}

int rc_launch_count(void *ctx, unsigned long long *out)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !out) return -1;
    *out = c->launches;
    return 0;
}


}  // extern "C"
