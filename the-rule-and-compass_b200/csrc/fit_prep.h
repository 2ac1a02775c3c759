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
    std::vector<FIns> fins;           /* per candidate: forward list | reverse list */
    std::vector<int> fins_off;        /* [P+1] */
    std::vector<int4> finfo;          /* forward count, reverse count, assembly threads,
                                         spill slots | tape slots << 16 */
    size_t asm_region = 0;            /* assembly shared region of the batch */
    int mmax = 1;                     /* most records */
    int pmax = 0;                     /* most constants */
    int fslots = 1;                   /* most spill slots */
    int ftape = 1;                    /* most tape slots */
    int fmaxins = 2;                  /* longest forward + reverse list */
};

/* Validate and translate `nprog` programs (`off` in words); a rejected
   program has valid[i] = 0 and no instructions. `extra_cols` widens the
   assembly's Gram beyond p + 1 columns (the correlation moments use 2). */
void prep_batch(const unsigned int *off, const unsigned int *prog, const int *pcount, int nprog,
                int v, FitPrep &b, int extra_cols = 0);
