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
 *    rows); each warp runs one candidate over all of its rows of the tile
 *    (features read from L2, where the whole matrix stays resident) and
 *    reduces once, and a hard failure ends the warp's rows of that candidate;
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
#include <fstream>
#include <map>
#include <mutex>
#include <numeric>
#include <vector>

#include "rc_internal.h"
#include "rc_ops.cuh"

#include "score_kernels.cuh"

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
       returns NaN for every row makes the program a single K_NAN. The
       instructions are written straight into `out` (at most one per word,
       so `nwords` of room; a word-free program needs one). */
    int n = 0;
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
            out[n++] = in;
        } else if (w == OP_HALT) {
            if (depth < 1) { ok = false; break; }
            in.kind = K_HALT;
            in.arg = depth == 1 ? 1 : 0;
            out[n++] = in;
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
            if (n > 0 && fusable(w)) {
                RcIns &prev = out[n - 1];
                if ((prev.kind == K_PUSH_VAR || prev.kind == K_PUSH_CONST) && prev.spill != 0xff &&
                    prev.spill == in.arg) {
                    uint8_t kind = prev.kind == K_PUSH_VAR ? K_BIN_V : K_BIN_C;
                    prev.kind = kind;
                    prev.op = (uint8_t)w;
                    prev.spill = 0xff;
                    continue;
                }
            }
            out[n++] = in;
        } else if (w == OP_IF) {
            if (depth < 3) { ok = false; break; }
            in.kind = K_IF;
            in.arg = (uint8_t)(depth - 3);
            depth -= 2;
            out[n++] = in;
        } else {
            /* Unary, including unknown codes, which evaluate to NaN
               (eval.cu:567). */
            if (depth < 1) { ok = false; break; }
            in.kind = K_UNARY;
            in.op = (uint8_t)(w > 255 ? 255 : w);
            if (w > 255 || w == OP_HALT) in.op = 254; /* unknown: NaN */
            out[n++] = in;
        }
    }
    if (!ok || !halted || n > RC_MAX_INS) {
        RcIns bad;
        memset(&bad, 0, sizeof(bad));
        bad.kind = K_NAN;
        bad.spill = 0xff;
        out[0] = bad;
        *nslots = 0;
        return 1;
    }
    *nslots = maxslot + 1;
    return n;
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

/* Rows per tile: fixed so a candidate's reduction order depends only on n
   and its own depth bucket. */
const int TILE_ROWS = RC_TILE_ROWS;
const int LANE_T = 128;

const void *score_kernel_fn(int T, bool track)
{
    if (T == 256) return track ? (const void *)rc_score_kernel<256, true>
                               : (const void *)rc_score_kernel<256, false>;
    return track ? (const void *)rc_score_kernel<64, true> : (const void *)rc_score_kernel<64, false>;
}

void launch_score_kernel(int T, bool track, int grid, size_t smem, cudaStream_t s,
                         const ScoreArgs &a)
{
    if (T == 256) {
        if (track) rc_score_kernel<256, true><<<grid, 256, smem, s>>>(a);
        else rc_score_kernel<256, false><<<grid, 256, smem, s>>>(a);
    } else {
        if (track) rc_score_kernel<64, true><<<grid, 64, smem, s>>>(a);
        else rc_score_kernel<64, false><<<grid, 64, smem, s>>>(a);
    }
}

/* The kernel's dynamic shared-memory limit raised to at least `smem`
   (monotone, shared with every other path: rc_raise_smem). */
int set_smem(const void *fn, size_t smem) { return rc_raise_smem(fn, smem); }

size_t lane_smem(int nslots) { return (size_t)nslots * LANE_T * 16 + RC_MAX_INS * sizeof(RcIns) + LANE_T * 8; }

}  // namespace


float rc_score_run(RcCtx *c, const uint32_t *words, const uint32_t *off, int width, int nprog,
                   int mode, const int *pcount, double *out, int *status, float *out_f32,
                   float *pred_out)
{
    (void)pcount;
    if (!c || nprog <= 0) return -1.0f;
    RcStats *st = &c->stats;
    const double t_begin = rc_now_ms();

    /* 1. decode, each program straight into its place (room for one
       instruction per word) */
    std::vector<int> ins_off(nprog + 1, 0);
    std::vector<int> nslots(nprog, 0);
    std::vector<int> opw(nprog, 0);
    size_t room = 0;
    for (int p = 0; p < nprog; ++p) {
        const size_t b = width > 0 ? (size_t)p * (size_t)width : off[p];
        const size_t e = width > 0 ? b + (size_t)width : off[p + 1];
        room += std::max<size_t>(e > b ? e - b : 0, 1);
    }
    std::vector<RcIns> ins(room);
    size_t pos = 0;
    for (int p = 0; p < nprog; ++p) {
        size_t b = width > 0 ? (size_t)p * (size_t)width : off[p];
        size_t e = width > 0 ? b + (size_t)width : off[p + 1];
        if (e < b) e = b;
        /* algorithmic ops of a row: postfix ops (a push counts one) + residual + loss */
        int ops = 0;
        for (size_t q = b; q < e && words[q] != OP_HALT; ++ops)
            q += (words[q] == OP_CONST || words[q] == OP_VAR) ? 2 : 1;
        opw[p] = ops + 2;
        int ns = 0;
        const int cnt = rc_decode_postfix(words + b, e - b, c->v, ins.data() + pos, &ns);
        ins_off[p] = (int)pos;
        pos += (size_t)cnt;
        nslots[p] = ns;
    }
    ins.resize(pos);
    ins_off[nprog] = (int)pos;

    /* 2. bucket by depth; longest program first */
    Bucket bk[2];
    int max_slots = 1;
    for (int p = 0; p < nprog; ++p) {
        const int b = nslots[p] <= RC_SHALLOW_SLOTS ? 0 : 1;
        bk[b].cands.push_back(p);
        bk[b].nslots = std::max(bk[b].nslots, nslots[p]);
        bk[b].maxins = std::max(bk[b].maxins, ins_off[p + 1] - ins_off[p]);
        max_slots = std::max(max_slots, nslots[p]);
    }
    /* longest program first, ties in slot order: a stable counting sort on
       the instruction count (1..RC_MAX_INS) */
    for (int b = 0; b < 2; ++b) {
        std::vector<int> &v = bk[b].cands;
        std::vector<int> at(RC_MAX_INS + 1, 0), sorted(v.size());
        auto key = [&](int x) {
            const int len = std::min(std::max(ins_off[x + 1] - ins_off[x], 1), RC_MAX_INS);
            return RC_MAX_INS - len;
        };
        for (int x : v) at[key(x) + 1]++;
        for (int k = 0; k < RC_MAX_INS; ++k) at[k + 1] += at[k];
        for (int x : v) sorted[at[key(x)]++] = x;
        v.swap(sorted);
    }
    const int Tb[2] = {256, 64};
    /* the scoring kernel reads features from L2; nothing is staged */
    const int staged = 0;
    const int ntiles = std::max(1, (c->n + TILE_ROWS - 1) / TILE_ROWS);
    std::vector<int> cand_tiles(nprog, ntiles);
    std::vector<int> order;
    order.reserve(nprog);
    for (int b = 0; b < 2; ++b) order.insert(order.end(), bk[b].cands.begin(), bk[b].cands.end());

    const bool corr = (mode == SM_CORRELATION || mode == SM_CORRELATION_SIGNED);
    const bool track = mode < SM_EVAL_SQUARED;

    /* 3. layout: inputs [ins | ins_off | order | cand_tiles], outputs
       [out | status | out_f32], work [part | bad | counters | pbar | lane]. */
    size_t cur = 0;
    const size_t o_ins = rc_take(&cur, sizeof(RcIns) * ins.size());
    const size_t o_insoff = rc_take(&cur, sizeof(int) * (nprog + 1));
    const size_t o_order = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_ctiles = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_opw = rc_take(&cur, sizeof(int) * nprog);
    const size_t in_end = rc_take(&cur, 0);
    const size_t o_out = rc_take(&cur, sizeof(double) * nprog);
    const size_t o_status = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_f32 = rc_take(&cur, sizeof(float) * nprog);
    const size_t o_rows = rc_take(&cur, 4 * sizeof(unsigned long long));
    const size_t io_end = rc_take(&cur, 0);
    const size_t o_part = rc_take(&cur, 4 * sizeof(double) * (size_t)nprog * ntiles);
    const size_t o_bad = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_bad64 = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_cnt = rc_take(&cur, sizeof(int) * 16);
    const size_t o_zero_end = rc_take(&cur, 0);
    const size_t o_pbar = rc_take(&cur, sizeof(double) * nprog);
    const size_t o_pbarerr = rc_take(&cur, sizeof(double) * nprog);
    const size_t o_pbar64 = rc_take(&cur, sizeof(double) * nprog);
    const size_t o_flagged = rc_take(&cur, sizeof(int) * nprog);
    const size_t o_badrow = rc_take(&cur, track && !corr ? sizeof(int) * nprog : 0);
    const size_t o_part64 = rc_take(&cur, track ? 2 * sizeof(double) * (size_t)nprog * ntiles : 0);
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
    memcpy(host + o_opw, opw.data(), sizeof(int) * nprog);
    cudaMemcpyAsync(dev, host, in_end, cudaMemcpyHostToDevice, c->s);
    cudaMemsetAsync(dev + o_bad, 0, o_zero_end - o_bad, c->s);
    cudaMemsetAsync(dev + o_rows, 0, 4 * sizeof(unsigned long long), c->s);
    unsigned long long *d_rows = reinterpret_cast<unsigned long long *>(dev + o_rows);
    if (track && !corr) cudaMemsetAsync(dev + o_badrow, 0x7f, sizeof(int) * nprog, c->s);
    st->h2d_ms += rc_now_ms() - t;
    st->h2d_bytes += in_end;

    int *d_cnt = reinterpret_cast<int *>(dev + o_cnt);
    int *d_nflag = d_cnt + 8;
    double *d_out = reinterpret_cast<double *>(dev + o_out);
    int *d_status = reinterpret_cast<int *>(dev + o_status);
    ScoreArgs a;
    memset(&a, 0, sizeof(a));
    a.cols = c->d_cols;
    a.y = c->d_y;
    a.tsign = c->d_tsign;
    a.w = c->d_w64;
    a.n = c->n;
    a.npad = c->npad;
    a.v = c->v;
    a.staged = staged;
    a.ins = reinterpret_cast<const RcIns *>(dev + o_ins);
    a.ins_off = reinterpret_cast<const int *>(dev + o_insoff);
    a.nprog = nprog;
    a.ptiles = ntiles;
    a.ntiles = ntiles;
    a.part = reinterpret_cast<double *>(dev + o_part);
    a.bad = reinterpret_cast<int *>(dev + o_bad);
    a.badrow = track && !corr ? reinterpret_cast<int *>(dev + o_badrow) : nullptr;
    a.rows = d_rows;
    a.opw = reinterpret_cast<const int *>(dev + o_opw);
    a.pred = pred_out ? reinterpret_cast<float *>(dev + o_pred) : nullptr;
    a.pbar = reinterpret_cast<const double *>(dev + o_pbar);
    a.pbar_err = reinterpret_cast<const double *>(dev + o_pbarerr);
    a.ybar = c->ybar;
    const int *d_ctiles = reinterpret_cast<const int *>(dev + o_ctiles);

    t = rc_now_ms();
    cudaEventRecord(c->t0, c->s);
    cudaEventRecord(c->sp[0], c->s);
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
            group = std::max(1, std::min(group, std::min(nb, 32)));
            a.order = reinterpret_cast<const int *>(dev + o_order) + obase;
            a.ncand = nb;
            a.group = group;
            a.subtiles = TILE_ROWS / (T * 4);
            const int ngroups = (nb + group - 1) / group;
            a.nitems = ngroups * ntiles;
            a.maxins = bk[b].maxins;
            a.nslots = std::max(bk[b].nslots, 1);
            a.counter = d_cnt + b + 2 * pass;
            a.mode = kmode;
            const size_t smem = T == 256
                ? ScoreSmem<256>::total(c->v, staged, a.nslots, group, a.maxins)
                : ScoreSmem<64>::total(c->v, staged, a.nslots, group, a.maxins);
            const void *fn = score_kernel_fn(T, track);
            if (set_smem(fn, smem) != 0) {
                st->failed = 1;
                cudaStreamSynchronize(c->s);
                return -1.0f;
            }
            int grid = c->sm_count * occupancy_blocks(fn, T, smem);
            if (grid > a.nitems) grid = a.nitems;
            launch_score_kernel(T, track, grid, smem, c->s, a);
            c->launches += 1;
            obase += nb;
        }
        if (pass == passes - 1) cudaEventRecord(c->sp[1], c->s);
        c->launches += 1;
        rc_score_finalize<<<(nprog + 127) / 128, 128, 0, c->s>>>(
            nprog, d_ctiles, a.part, ntiles, a.bad, c->n, (corr && pass == 1) ? mode : kmode,
            c->syy, d_out, d_status,
            reinterpret_cast<float *>(dev + o_f32), reinterpret_cast<double *>(dev + o_pbar),
            reinterpret_cast<double *>(dev + o_pbarerr), d_nflag,
            track ? reinterpret_cast<int *>(dev + o_flagged) : nullptr);
    }

    /* 4. the f64 re-check lane over the flagged candidates */
    if (track) {
        Score64Args l;
        memset(&l, 0, sizeof(l));
        l.cols = c->d_cols;
        l.y = c->d_y;
        l.tsign = c->d_tsign;
        l.w = c->d_w64;
        l.n = c->n;
        l.npad = c->npad;
        l.ins = a.ins;
        l.ins_off = a.ins_off;
        l.flagged = reinterpret_cast<const int *>(dev + o_flagged);
        l.nflag = d_nflag;
        l.ntiles = ntiles;
        l.nslots = max_slots;
        l.part = reinterpret_cast<double *>(dev + o_part64);
        l.nprog = nprog;
        l.ptiles = ntiles;
        l.bad = reinterpret_cast<int *>(dev + o_bad64);
        l.pbar = reinterpret_cast<const double *>(dev + o_pbar64);
        l.ybar = c->ybar;
        l.rows = d_rows + 1;
        l.opw = a.opw;
        const size_t smem = lane_smem(max_slots);
        if (set_smem((const void *)rc_score64_kernel<LANE_T>, smem) != 0) {
            st->failed = 1;
            cudaStreamSynchronize(c->s);
            return -1.0f;
        }
        const int grid = c->sm_count *
                         occupancy_blocks((const void *)rc_score64_kernel<LANE_T>, LANE_T, smem);
        if (a.badrow) {
            /* the f32 failure rows first: most failures are confirmed there */
            l.mode = mode;
            const size_t csmem = (size_t)max_slots * 32 * 16 + RC_MAX_INS * sizeof(RcIns);
            if (set_smem((const void *)rc_badrow_check<32>, csmem) != 0) {
                st->failed = 1;
                cudaStreamSynchronize(c->s);
                return -1.0f;
            }
            rc_badrow_check<32><<<nprog, 32, csmem, c->s>>>(l, a.badrow);
            c->launches += 1;
        }
        for (int pass = 0; pass < passes; ++pass) {
            const int kmode = corr ? (pass == 0 ? SM_CORR_PASS1 : SM_CORR_PASS2) : mode;
            if (pass == 1) cudaMemsetAsync(dev + o_bad64, 0, sizeof(int) * nprog, c->s);
            l.counter = d_cnt + 4 + pass;
            l.mode = kmode;
            c->launches += 2;
            rc_score64_kernel<LANE_T><<<grid, LANE_T, smem, c->s>>>(l);
            rc_score64_finalize<<<(nprog + 127) / 128, 128, 0, c->s>>>(
                l.flagged, d_nflag, ntiles, l.part, nprog, ntiles, l.bad, c->n,
                (corr && pass == 1) ? mode : kmode, c->syy,
                d_out, d_status, reinterpret_cast<double *>(dev + o_pbar64));
        }
    }
    cudaEventRecord(c->sp[2], c->s);
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
    memcpy(c->prof_rows, host + o_rows, sizeof(c->prof_rows));
    memcpy(c->prof_ops, host + o_rows + 2 * sizeof(unsigned long long), sizeof(c->prof_ops));
    c->prof_ms[0] = c->prof_ms[1] = 0.0f;
    cudaEventElapsedTime(&c->prof_ms[0], c->sp[0], c->sp[1]);
    cudaEventElapsedTime(&c->prof_ms[1], c->sp[1], c->sp[2]);
    c->prof_valid = 1;
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
        if (c->pool_host[i].assign((size_t)nprog * width, (uint32_t)OP_HALT) != 0) {
            c->stats.failed = 1;
            return -1;
        }
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
    c->launches += 1;
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
                                  int *__restrict__ deep, int *__restrict__ ins_len, int ntiles)
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
    ins_len[p] = n;
    if (!ok || !halted || maxslot + 1 > RC_SHALLOW_SLOTS) {
        deep[p] = ok && halted ? 1 : 0;
        RcIns bad;
        bad.kind = K_NAN;
        bad.op = 0;
        bad.arg = 0;
        bad.spill = 0xff;
        bad.imm = 0;
        out[0] = bad;
        ins_len[p] = 1;
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
    int lane_per_sm;
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
    const size_t o_len = rc_take(&cur, sizeof(int) * (size_t)nprog);
    const size_t o_part = rc_take(&cur, 4 * sizeof(double) * (size_t)nprog * ntiles);
    const size_t o_part64 = rc_take(&cur, 2 * sizeof(double) * (size_t)nprog * ntiles);
    const size_t o_flagged = rc_take(&cur, sizeof(int) * (size_t)nprog);
    const size_t o_bad = rc_take(&cur, sizeof(int) * (size_t)nprog);
    const size_t o_bad64 = rc_take(&cur, sizeof(int) * (size_t)nprog);
    const size_t o_cnt = rc_take(&cur, sizeof(int) * 16);
    const size_t o_zero_end = rc_take(&cur, 0);
    const size_t need = rc_take(&cur, 0);
    if (need > RC_NOALLOC_SCRATCH_BYTES) {
        fprintf(stderr,
                "rc_score_batch_noalloc: %d programs over %d rows need %zu scratch bytes, the "
                "static maximum is %u\n",
                nprog, n, need, RC_NOALLOC_SCRATCH_BYTES);
        return -2;
    }
    const int G = 8;
    const int group = G < nprog ? G : nprog;
    /* features are read from global memory (L2), nothing is staged */
    const size_t smem = ScoreSmem<256>::total(v, 0, RC_SHALLOW_SLOTS, group, RC_MAX_INS);
    const size_t lsmem = lane_smem(RC_SHALLOW_SLOTS);
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
            const size_t maxsmem = ScoreSmem<256>::total(0, 0, RC_SHALLOW_SLOTS, G, RC_MAX_INS);
            if (set_smem((const void *)rc_score_kernel<256, true>, maxsmem) != 0 ||
                set_smem((const void *)rc_score64_kernel<LANE_T>, lsmem) != 0)
                return -1;
            int sms = 1;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            d->scratch = (unsigned char *)ptr;
            d->sm_count = sms > 0 ? sms : 1;
            d->grid_per_sm =
                occupancy_blocks((const void *)rc_score_kernel<256, true>, T, maxsmem);
            d->lane_per_sm =
                occupancy_blocks((const void *)rc_score64_kernel<LANE_T>, LANE_T, lsmem);
            d->ready = 1;
        }
    }
    /* the limits only grow, and another path may have launched these
       kernels since; raising them again is a no-op when already high enough */
    if (set_smem((const void *)rc_score_kernel<256, true>, smem) != 0 ||
        set_smem((const void *)rc_score64_kernel<LANE_T>, lsmem) != 0) {
        fprintf(stderr, "rc_score_batch_noalloc: cannot raise the shared-memory limit\n");
        return -1;
    }
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char *sc = d->scratch;
    cudaMemsetAsync(sc + o_bad, 0, o_zero_end - o_bad, s);
    rc_noalloc_decode<<<(nprog + 1 + 127) / 128, 128, 0, s>>>(
        prog, off, nprog, v, reinterpret_cast<RcIns *>(sc + o_ins),
        reinterpret_cast<int *>(sc + o_insoff), reinterpret_cast<int *>(sc + o_order),
        reinterpret_cast<int *>(sc + o_ctiles), reinterpret_cast<int *>(sc + o_deep),
        reinterpret_cast<int *>(sc + o_len), ntiles);
    int *cnt = reinterpret_cast<int *>(sc + o_cnt);
    ScoreArgs a;
    memset(&a, 0, sizeof(a));
    a.cols = cols;
    a.y = y;
    a.n = n;
    a.npad = ld;
    a.v = v;
    a.staged = 0;
    a.ins = reinterpret_cast<const RcIns *>(sc + o_ins);
    a.ins_off = reinterpret_cast<const int *>(sc + o_insoff);
    a.ins_len = reinterpret_cast<const int *>(sc + o_len);
    a.order = reinterpret_cast<const int *>(sc + o_order);
    a.ncand = nprog;
    a.group = group;
    a.subtiles = TILE_ROWS / SUB;
    a.ntiles = ntiles;
    a.nitems = ((nprog + a.group - 1) / a.group) * ntiles;
    a.maxins = RC_MAX_INS;
    a.nslots = RC_SHALLOW_SLOTS;
    a.counter = cnt;
    a.part = reinterpret_cast<double *>(sc + o_part);
    a.nprog = nprog;
    a.ptiles = ntiles;
    a.bad = reinterpret_cast<int *>(sc + o_bad);
    a.mode = kind;
    int grid = d->sm_count * d->grid_per_sm;
    if (grid > a.nitems) grid = a.nitems;
    rc_score_kernel<256, true><<<grid, T, smem, s>>>(a);
    {
        /* a failed scoring launch must not let the finalize kernels write
           stale scratch into the caller's outputs */
        const cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) {
            fprintf(stderr, "rc_score_batch_noalloc: scoring launch failed: %s\n",
                    cudaGetErrorString(le));
            return -1;
        }
    }
    rc_score_finalize<<<(nprog + 127) / 128, 128, 0, s>>>(
        nprog, reinterpret_cast<const int *>(sc + o_ctiles), a.part, ntiles, a.bad, n, kind, 0.0,
        out, status, nullptr, nullptr, nullptr, cnt + 8, reinterpret_cast<int *>(sc + o_flagged));
    Score64Args l;
    memset(&l, 0, sizeof(l));
    l.cols = cols;
    l.y = y;
    l.n = n;
    l.npad = ld;
    l.ins = a.ins;
    l.ins_off = a.ins_off;
    l.flagged = reinterpret_cast<const int *>(sc + o_flagged);
    l.nflag = cnt + 8;
    l.ntiles = ntiles;
    l.nslots = RC_SHALLOW_SLOTS;
    l.counter = cnt + 4;
    l.part = reinterpret_cast<double *>(sc + o_part64);
    l.nprog = nprog;
    l.ptiles = ntiles;
    l.bad = reinterpret_cast<int *>(sc + o_bad64);
    l.mode = kind;
    rc_score64_kernel<LANE_T><<<d->sm_count * d->lane_per_sm, LANE_T, lsmem, s>>>(l);
    rc_score64_finalize<<<(nprog + 127) / 128, 128, 0, s>>>(l.flagged, l.nflag, ntiles, l.part,
                                                            nprog, ntiles, l.bad, n, kind, 0.0,
                                                            out, status, nullptr);
    rc_noalloc_mark_deep<<<(nprog + 127) / 128, 128, 0, s>>>(
        nprog, reinterpret_cast<const int *>(sc + o_deep), out, status);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "rc_score_batch_noalloc: launch failed: %s\n", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

/* Profile of the context's last scoring call: device ms of the f32 scoring
   kernels (from the first scoring launch to the end of the last one) and of
   everything after them (finalize, the f64 lane and its finalize), and the
   rows each interpreter evaluated (a candidate stops at its first hard
   failure, so these can be below candidates x rows), and those rows weighted
   by their candidate's postfix ops + 2 (the algorithmic lane-ops). */
extern "C" int rc_last_score_profile(void *ctx, float *ms_f32, float *ms_rest,
                                     unsigned long long *rows_f32,
                                     unsigned long long *rows_f64,
                                     unsigned long long *ops_f32, unsigned long long *ops_f64)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !c->prof_valid) return -1;
    if (ms_f32) *ms_f32 = c->prof_ms[0];
    if (ms_rest) *ms_rest = c->prof_ms[1];
    if (rows_f32) *rows_f32 = c->prof_rows[0];
    if (rows_f64) *rows_f64 = c->prof_rows[1];
    if (ops_f32) *ops_f32 = c->prof_ops[0];
    if (ops_f64) *ops_f64 = c->prof_ops[1];
    return 0;
}

/* ---- launch-shape autotuner ------------------------------------------- */

/* Candidates per work item (the group G) for each length bucket, chosen by
   timing the scorer on the caller's batch: per bucket, every G in
   {1, 2, 4, 8, 16, 32} is run three times after a warm-up on that bucket's
   programs and the fastest median kept in the context. With a path, entries
   for this (N, V) are read first (a bucket found there is not re-timed) and
   the table is written back as lines "n v bucket group". */
extern "C" int rc_autotune(void *ctx, const unsigned int *prog, const unsigned int *off, int nprog,
                           const char *path)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !prog || !off || nprog <= 0) return -1;
    std::vector<int> have(2, 0);
    std::vector<std::string> keep;
    if (path) {
        std::ifstream in(path);
        long long n, v;
        int b, g;
        std::string line;
        while (std::getline(in, line)) {
            if (sscanf(line.c_str(), "%lld %lld %d %d", &n, &v, &b, &g) != 4) continue;
            if (n == c->n && v == c->v && b >= 0 && b < 2 && g >= 1 && g <= 32) {
                c->tune[b] = std::make_pair(g, 0);
                have[b] = 1;
            } else {
                keep.push_back(line);
            }
        }
    }
    /* split the batch by bucket */
    std::vector<uint32_t> words[2], offs[2];
    offs[0].push_back(0);
    offs[1].push_back(0);
    std::vector<RcIns> tmp;
    for (int i = 0; i < nprog; ++i) {
        int ns = 0;
        /* (room for one instruction per word) */
        tmp.resize(std::max<size_t>(off[i + 1] > off[i] ? off[i + 1] - off[i] : 0, 1));
        const int cnt = rc_decode_postfix(prog + off[i], off[i + 1] - off[i], c->v, tmp.data(), &ns);
        if (cnt <= 0) continue;
        const int b = ns <= RC_SHALLOW_SLOTS ? 0 : 1;
        words[b].insert(words[b].end(), prog + off[i], prog + off[i + 1]);
        offs[b].push_back((uint32_t)words[b].size());
    }
    for (int b = 0; b < 2; ++b) {
        const int nb = (int)offs[b].size() - 1;
        if (nb == 0 || have[b]) continue;
        std::vector<double> out(nb);
        std::vector<int> status(nb), pc(nb, 0);
        std::vector<float> f32(nb);
        int best_g = 8;
        float best = 1e30f;
        for (int g = 1; g <= 32; g *= 2) {
            c->tune[b] = std::make_pair(g, 0);
            float t[4];
            bool ok = true;
            for (int r = 0; r < 4 && ok; ++r) {
                t[r] = rc_score_run(c, words[b].data(), offs[b].data(), 0, nb, SM_SQUARED, pc.data(),
                                    out.data(), status.data(), f32.data(), nullptr);
                ok = t[r] >= 0.0f;
            }
            if (!ok) continue;
            std::sort(t + 1, t + 4);
            if (t[2] < best) {
                best = t[2];
                best_g = g;
            }
        }
        c->tune[b] = std::make_pair(best_g, 0);
    }
    if (path) {
        std::ofstream o(path, std::ios::trunc);
        for (const std::string &l : keep) o << l << "\n";
        for (const auto &kv : c->tune)
            o << c->n << " " << c->v << " " << kv.first << " " << kv.second.first << "\n";
        if (!o) return -1;
    }
    return (int)c->tune.size();
}
