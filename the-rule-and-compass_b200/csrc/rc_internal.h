/*
 * Host-side internals of librcsr_b200: the context, its growable device and
 * pinned regions, and the decoded scoring program format.
 */
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "rcsr_b200.h"

/* Device rows are padded to a multiple of this many rows so that every
   scoring sub-tile reads whole, 16-byte aligned float4 groups. */
#define RC_ROW_PAD 4096

/* ---- decoded scoring programs ----------------------------------------
 *
 * The postfix words of the reference format are translated once per batch on
 * the host into 8-byte instructions for a top-of-stack-in-registers machine:
 * the top of stack lives in registers (four rows per thread), deeper entries
 * in per-thread shared-memory slots whose index is fixed at decode time, and a
 * push immediately consumed by a binary operator is fused into it. */
enum RcInsKind {
    K_PUSH_VAR = 0,   /* spill TOS to slot `spill` (0xff: none); TOS = x[imm] */
    K_PUSH_CONST = 1, /* spill TOS; TOS = imm */
    K_UNARY = 2,      /* TOS = op(TOS) */
    K_BIN_S = 3,      /* TOS = op(slot[arg], TOS) */
    K_BIN_V = 4,      /* TOS = op(TOS, x[imm]) */
    K_BIN_C = 5,      /* TOS = op(TOS, imm) */
    K_IF = 6,         /* TOS = slot[arg] > 0 ? slot[arg + 1] : TOS */
    K_HALT = 7,       /* result = TOS (depth 1) or slot[0] (depth > 1) */
    K_NAN = 8         /* the whole program is a hard failure (NaN every row) */
};

struct RcIns {
    uint8_t kind;
    uint8_t op;
    uint8_t arg;   /* stack slot (K_BIN_S, K_IF), depth flag (K_HALT) */
    uint8_t spill; /* slot the TOS spills to on a push, 0xff when the stack is empty */
    uint32_t imm;  /* f32 bits of a constant, or a variable column */
};
static_assert(sizeof(RcIns) == 8, "RcIns is 8 bytes");

/* Deepest spill slot a shallow-bucket program may use (slots 0..14). */
#define RC_SHALLOW_SLOTS 15
/* Instructions per program the scoring kernel stages (HALT included). The
   postfix format allows at most 64 stack entries; a program longer than this
   is scored by splitting nothing -- it is rejected as a hard failure. */
#define RC_MAX_INS 256

/* Decode one postfix program (words [begin, end)). Returns the instruction
   count, fills `nslots` with the number of spill slots it uses, and emits a
   single K_NAN instruction for a program the device must score as NaN on
   every row (stack under/overflow, a missing HALT, a variable column >= v,
   or a program longer than RC_MAX_INS). `out` needs room for max(nwords, 1)
   instructions (at most one per word is written). */
int rc_decode_postfix(const uint32_t *words, size_t nwords, int v, RcIns *out, int *nslots);

/* ---- context ---------------------------------------------------------- */

struct RcPending {
    int active;
    int nprog;
    int loss;
    cudaEvent_t done;
};

/* A page-locked host array of words: device-to-host copies into it run at
   full speed and need no staging. */
struct RcPinnedWords {
    uint32_t *p = nullptr;
    size_t n = 0;
    uint32_t *data() { return p; }
    const uint32_t *data() const { return p; }
    /* `count` words, all `v` (reallocated when larger); 0, or -1 when the
       allocation fails (the array is then empty). */
    int assign(size_t count, uint32_t v)
    {
        if (count > n) {
            release();
            if (cudaHostAlloc((void **)&p, sizeof(uint32_t) * (count ? count : 1),
                              cudaHostAllocPortable) != cudaSuccess) {
                cudaGetLastError();
                p = nullptr;
                return -1;
            }
            n = count;
        }
        for (size_t i = 0; i < count; ++i) p[i] = v;
        return 0;
    }
    void release()
    {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
    }
    RcPinnedWords() = default;
    RcPinnedWords(const RcPinnedWords &) = delete;
    RcPinnedWords &operator=(const RcPinnedWords &) = delete;
    ~RcPinnedWords() { release(); }
};

struct RcCtx {
    int n;      /* rows */
    int v;      /* columns */
    int npad;   /* padded row stride of the device columns */
    int device;
    int sm_count;
    float *d_cols;   /* [v][npad] f32, zero padded */
    float *d_y;      /* [npad] */
    double *d_cols64; /* [v][npad] f64 twins (rc_set_fit_data, or a cast) */
    double *d_y64;
    double *d_w64;    /* [npad] base row weights, NULL when unweighted */
    float *d_tsign;
    double *d_tsign64;
    int has_tsign;
    int fit_data_exact; /* 1 when the f64 twins came from rc_set_fit_data */
    double ybar, syy;

    cudaStream_t s;
    cudaEvent_t t0, t1, ev_done;

    /* growable per-call regions */
    unsigned char *dev;
    size_t dev_bytes;
    unsigned char *host;
    size_t host_bytes;

    /* staged postfix batch (rc_set_programs) */
    std::vector<uint32_t> prog_words;
    std::vector<uint32_t> prog_off;
    int nprog;

    /* fixed-stride pool (host mirrors page-locked: the new pool comes back
       every generation) */
    RcPinnedWords pool_host[2];
    unsigned int *d_pool[2];
    int pool_cap;
    int pool_width;

    RcPending pending;

    /* rank target cache */
    long long *d_rank_b;
    int rank_ready;
    unsigned long long rank_bb[2];
    /* rank sums: bucket capacity (0 = built in, -1 = radix sort only), the
       largest group of distinct keys ranked by comparison (0 = built in),
       and the segments of the last call that took the radix sort */
    int rank_cap;
    int rank_gmax;
    int rank_fallbacks;

    /* ledger and arena accounting */
    RcStats stats;
    double batch_start_ms;
    int async_copy;
    char sync_reason[96];
    unsigned long long alloc_calls;
    unsigned long long steady_alloc_calls;
    unsigned long long batches;
    unsigned long long fs_growths;
    int warm;

    /* autotuned scoring shapes: key = (bucket) -> (group, subtiles) */
    std::map<int, std::pair<int, int>> tune;
    /* autotuned fit assembly budget (KB) per length bucket, 0 = default */
    int fit_budget_kb[4];

    /* cached CUDA graph of the fused fit for a repeated batch shape */
    cudaGraphExec_t fit_graph;
    std::string fit_graph_key;
    std::string fit_seen_key;             /* the last batch shape run without a graph */
    unsigned long long fit_graph_kernels; /* kernel nodes in one replay */

    /* kernels this context has launched (graph replays count their nodes) */
    unsigned long long launches;

    /* the last fit's per-candidate state, in the device region (for
       rc_last_fit_sweeps; valid until the region is reused) */
    unsigned char *fit_state;
    int fit_state_n;
    size_t fit_state_stride;

    /* profile of the last scoring call (rc_last_score_profile): events
       around the f32 scoring kernels and the f64 lane, rows evaluated */
    cudaEvent_t sp[3];
    unsigned long long prof_rows[2];
    unsigned long long prof_ops[2];
    float prof_ms[2];
    int prof_valid;
};

double rc_now_ms();
/* Grow the per-call device / pinned regions (high-water mark, counted). */
int rc_reserve(RcCtx *c, size_t dev_bytes, size_t host_bytes);
size_t rc_take(size_t *cur, size_t bytes);
/* Raise a kernel's dynamic shared-memory limit on the current device to at
   least `bytes`; the limit only ever grows (shared by every context and
   path). Returns 0, or -1 when the device refuses the size. */
int rc_raise_smem(const void *fn, size_t bytes);
/* Make sure the f64 twins exist (cast from the f32 rows when the caller never
   uploaded exact rows). */
int rc_ensure_f64(RcCtx *c);
/* Stream-ordered event synchronisation of the context's stream. */
int rc_finish(RcCtx *c);

/* Scoring entry used by rc_score_batch / rc_pool_score / rc_eval / rc_predict.
   `mode` is an internal scoring mode (see score.cu). Results are written to
   the host buffers. Returns kernel ms or a negative value. */
float rc_score_run(RcCtx *c, const uint32_t *words, const uint32_t *off, int width, int nprog,
                   int mode, const int *pcount, double *out, int *status, float *out_f32,
                   float *pred_out);
