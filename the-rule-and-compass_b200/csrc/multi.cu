/*
 * Several GPUs behind one handle: candidate sharding through the C ABI.
 *
 * The device path shards by candidate: every program is independent given
 * the resident rows, so each GPU keeps its own copy of the rows (its own
 * context) and serves a contiguous slice of the batch; the per-candidate
 * outputs land in the caller's arrays at the slice's offset. No data-path
 * collective is needed (the reference's island search is one process; this is
 * the additive multi-GPU form a C or Rust caller can bind). One host thread
 * per device makes that device current, calls the single-device entry point
 * on its slice and joins; the call returns the slowest slice's device ms.
 *
 * Slices are balanced by program words (a fair proxy of interpreter work),
 * and a candidate's results do not depend on which slice holds it, so a
 * sharded batch answers bit for bit what one context would.
 */
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "rc_internal.h"

extern "C" {
void *rc_create(const float *cols, int n, int v, const float *y);
void rc_destroy(void *ctx);
int rc_set_fit_data(void *ctx, const double *cols, const double *y, const double *w);
float rc_score_batch(void *ctx, const unsigned int *prog, const unsigned int *off, int nprog,
                     int kind, const int *pcount, double *out, int *status);
float rc_fit_batch_fused(void *ctx, const unsigned int *prog, const unsigned int *off,
                         const int *pcount, int nprog, int kmax, const double *c0,
                         const int *gauge, int iters, int metric, int flags, double *outc,
                         double *outsse, int *outstatus);
}

namespace {

struct RcMulti {
    std::vector<int> dev;
    std::vector<void *> ctx;
};

/* Contiguous slices [cut[d], cut[d + 1]) of nprog programs with about equal
   program words each. */
std::vector<int> balance(const unsigned int *off, int nprog, int nd)
{
    std::vector<int> cut(nd + 1, nprog);
    cut[0] = 0;
    const double total = (double)(off[nprog] - off[0]);
    int i = 0;
    for (int d = 1; d < nd; ++d) {
        const double goal = total * d / nd;
        while (i < nprog && (double)(off[i] - off[0]) < goal) ++i;
        cut[d] = i;
    }
    for (int d = 1; d <= nd; ++d) cut[d] = std::max(cut[d], cut[d - 1]);
    return cut;
}

/* Run `fn(d)` on one host thread per device with that device current; the
   results are combined by the caller. */
template <typename F>
void on_devices(const RcMulti *m, F fn)
{
    std::vector<std::thread> th;
    for (size_t d = 0; d < m->dev.size(); ++d)
        th.emplace_back([m, d, &fn]() {
            if (cudaSetDevice(m->dev[d]) != cudaSuccess) {
                cudaGetLastError();
                fn((int)d, false);
                return;
            }
            fn((int)d, true);
        });
    for (auto &t : th) t.join();
}

/* A slice's rebased offsets off[lo..hi] - off[lo]. */
std::vector<unsigned int> rebase(const unsigned int *off, int lo, int hi)
{
    std::vector<unsigned int> o(hi - lo + 1);
    for (int i = lo; i <= hi; ++i) o[i - lo] = off[i] - off[lo];
    return o;
}

}  // namespace

extern "C" {

/* One context per device in `devices` (ndev of them; the same device may be
   named twice), each holding the rows. NULL on failure. */
void *rc_multi_create(const float *cols, int n, int v, const float *y, int ndev,
                      const int *devices)
{
    if (ndev <= 0 || !devices) return nullptr;
    RcMulti *m = new (std::nothrow) RcMulti();
    if (!m) return nullptr;
    m->dev.assign(devices, devices + ndev);
    m->ctx.assign(ndev, nullptr);
    on_devices(m, [&](int d, bool ok) {
        if (ok) m->ctx[d] = rc_create(cols, n, v, y);
    });
    for (void *c : m->ctx)
        if (!c) {
            on_devices(m, [&](int d, bool ok) {
                if (ok && m->ctx[d]) rc_destroy(m->ctx[d]);
            });
            delete m;
            return nullptr;
        }
    return m;
}

void rc_multi_destroy(void *h)
{
    RcMulti *m = (RcMulti *)h;
    if (!m) return;
    on_devices(m, [&](int d, bool ok) {
        if (ok && m->ctx[d]) rc_destroy(m->ctx[d]);
    });
    delete m;
}

/* rc_set_fit_data on every device. */
int rc_multi_set_fit_data(void *h, const double *cols, const double *y, const double *w)
{
    RcMulti *m = (RcMulti *)h;
    if (!m) return -1;
    std::vector<int> rc(m->dev.size(), -1);
    on_devices(m, [&](int d, bool ok) {
        if (ok) rc[d] = rc_set_fit_data(m->ctx[d], cols, y, w);
    });
    for (int r : rc)
        if (r != 0) return -1;
    return 0;
}

/* rc_score_batch over the devices: contiguous slices of the batch, outputs
   in place. Returns the slowest slice's kernel ms, or -1 if any slice
   failed (every output is then to be discarded). */
float rc_multi_score_batch(void *h, const unsigned int *prog, const unsigned int *off, int nprog,
                           int kind, const int *pcount, double *out, int *status)
{
    RcMulti *m = (RcMulti *)h;
    if (!m || !prog || !off || nprog <= 0 || !out || !status) return -1.0f;
    const int nd = (int)m->dev.size();
    const std::vector<int> cut = balance(off, nprog, nd);
    std::vector<float> ms(nd, 0.0f);
    on_devices(m, [&](int d, bool ok) {
        const int lo = cut[d], hi = cut[d + 1];
        if (hi <= lo) return;
        if (!ok) {
            ms[d] = -1.0f;
            return;
        }
        const std::vector<unsigned int> o = rebase(off, lo, hi);
        ms[d] = rc_score_batch(m->ctx[d], prog + off[lo], o.data(), hi - lo, kind,
                               pcount ? pcount + lo : nullptr, out + lo, status + lo);
    });
    float worst = 0.0f;
    for (float t : ms) {
        if (t < 0.0f) return -1.0f;
        worst = std::max(worst, t);
    }
    return worst;
}

/* rc_fit_batch_fused over the devices, sliced the same way. */
float rc_multi_fit_batch(void *h, const unsigned int *prog, const unsigned int *off,
                         const int *pcount, int nprog, int kmax, const double *c0,
                         const int *gauge, int iters, int metric, int flags, double *outc,
                         double *outsse, int *outstatus)
{
    RcMulti *m = (RcMulti *)h;
    if (!m || !prog || !off || !pcount || !c0 || nprog <= 0 || kmax <= 0 || !outc || !outsse ||
        !outstatus)
        return -1.0f;
    const int nd = (int)m->dev.size();
    const std::vector<int> cut = balance(off, nprog, nd);
    std::vector<float> ms(nd, 0.0f);
    on_devices(m, [&](int d, bool ok) {
        const int lo = cut[d], hi = cut[d + 1];
        if (hi <= lo) return;
        if (!ok) {
            ms[d] = -1.0f;
            return;
        }
        const std::vector<unsigned int> o = rebase(off, lo, hi);
        ms[d] = rc_fit_batch_fused(m->ctx[d], prog + off[lo], o.data(), pcount + lo, hi - lo,
                                   kmax, c0 + (size_t)lo * kmax, gauge ? gauge + 2 * lo : nullptr,
                                   iters, metric, flags, outc + (size_t)lo * kmax, outsse + lo,
                                   outstatus + lo);
    });
    float worst = 0.0f;
    for (float t : ms) {
        if (t < 0.0f) return -1.0f;
        worst = std::max(worst, t);
    }
    return worst;
}

/* The number of devices of a handle, and each device's context (for the
   single-device calls: make that device current first). */
int rc_multi_devices(void *h, void **ctx_out)
{
    RcMulti *m = (RcMulti *)h;
    if (!m) return -1;
    if (ctx_out)
        for (size_t d = 0; d < m->ctx.size(); ++d) ctx_out[d] = m->ctx[d];
    return (int)m->ctx.size();
}

}  // extern "C"
