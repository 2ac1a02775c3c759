/*
 * Host-side decode of a batch of fit-record programs (my-version/src/fit.rs
 * :985-1056 records) for the device sweeps: validation, the stack-machine
 * instruction lists and the per-candidate shapes. Shared by the fit and the
 * exact-statistics entry points.
 */
#pragma once

#include <vector>

#include "fit_interp.cuh"

struct FitPrep {
    std::vector<int> node_off, valid; /* record offsets [P+1]; 1 = accepted */
    std::vector<int> ninternal;       /* per candidate: records that are not leaves */
    std::vector<FIns> fins;           /* per candidate: forward list | reverse list */
    std::vector<int> fins_off;        /* [P+1] */
    std::vector<int4> finfo;          /* forward count, reverse count, assembly threads |
                                         launch class << 16, spill slots | tape slots << 16 */
    size_t asm_region = 0;            /* assembly shared region of the batch */
    size_t asm_reg[6] = {256, 256, 256, 256, 256, 256}; /* ... of each assembly launch class */
    int nclass[6] = {0, 0, 0, 0, 0, 0}; /* candidates of each assembly launch class */
    int mmax = 1;                     /* most records */
    int pmax = 0;                     /* most constants */
    int fslots = 1;                   /* most spill slots */
    int ftape = 1;                    /* most tape slots */
    int fmaxins = 2;                  /* longest forward + reverse list */

    /* constant-free subtree cache (requested by prep_batch's cache_npad) */
    std::vector<int2> fcinfo;         /* per candidate: cached forward count (the list
                                         follows the reverse list), first cache column */
    std::vector<FIns> sub_fins;       /* forward lists of the cached subtrees */
    std::vector<int> sub_off;         /* [nsub + 1] */
    std::vector<int> sub_col;         /* [nsub] cache column of each subtree */
    std::vector<int> sub_cand_off;    /* [P + 1] first subtree of each candidate */
    int ncache = 0;                   /* cache columns */
    int sub_slots = 1;                /* most spill slots of a subtree program */
    int sub_maxins = 2;               /* longest subtree program */
};

/* Validate and translate `nprog` programs (`off` in words); a rejected
   program has valid[i] = 0 and no instructions. `extra_cols` widens the
   assembly's Gram beyond p + 1 columns (the correlation moments use 2).
   With cache_bytes_per_col > 0, constant-free subtrees are cached (columns of
   that many bytes) while the total stays within cache_cap bytes; later
   candidates keep their full forward list. `bucket_budget_kb` (4 entries,
   0 = the default) is the assembly region budget of each length bucket,
   which sets a candidate's active threads. */
void prep_batch(const unsigned int *off, const unsigned int *prog, const int *pcount, int nprog,
                int v, FitPrep &b, int extra_cols = 0, size_t cache_bytes_per_col = 0,
                size_t cache_cap = 0, const int *bucket_budget_kb = nullptr);
