/*
 * The device context: resident rows, one non-blocking stream, growable
 * device / pinned per-call regions, telemetry.
 *
 * Mirrors the reference's context lifecycle and accounting
 * (my-version/src/cuda/eval.cu:89-391 `RcCtx`, :2721-2885 the persistent
 * regions, :3137-3266 rc_create/rc_destroy, :3836-3861 the ledger,
 * :3469-3512 the arena report). Rows are stored column-major and padded to
 * RC_ROW_PAD rows so every kernel reads whole aligned float4/double2 groups.
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "rc_internal.h"

double rc_now_ms()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec * 1e3 + (double)ts.tv_nsec / 1e6;
}

/* Raise a kernel's dynamic shared-memory limit on the current device to at
   least `bytes`. The limit only ever grows: every path and context that
   launches the kernel on the device shares it, and lowering it for a small
   launch would make a larger one (queued by another context, or held in a
   captured graph) fail. It is never set below 48 KB (the default a launch
   that needs no raise relies on), so a kernel with static shared memory
   gets room for both. Returns 0, or -1 when the device refuses the size. */
int rc_raise_smem(const void *fn, size_t bytes)
{
    bytes = std::max(bytes, (size_t)48 * 1024);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> raised;
    std::lock_guard<std::mutex> lock(mu);
    size_t &cur = raised[std::make_pair(fn, dev)];
    if (bytes <= cur) return 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
        cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    cur = bytes;
    return 0;
}

size_t rc_take(size_t *cur, size_t bytes)
{
    size_t o = (*cur + 255) & ~(size_t)255;
    *cur = o + bytes;
    return o;
}

int rc_reserve(RcCtx *c, size_t dev_bytes, size_t host_bytes)
{
    /* every call reuses the region: the last fit's state is gone */
    c->fit_state = nullptr;
    c->fit_state_n = 0;
    if (dev_bytes < 256) dev_bytes = 256;
    if (host_bytes < 256) host_bytes = 256;
    if (dev_bytes > c->dev_bytes) {
        if (c->dev) {
            cudaStreamSynchronize(c->s);
            cudaFree(c->dev);
            c->dev = nullptr;
            c->dev_bytes = 0;
        }
        size_t want = dev_bytes + dev_bytes / 4;
        void *p = nullptr;
        if (cudaMalloc(&p, want) != cudaSuccess) {
            cudaGetLastError();
            want = dev_bytes;
            if (cudaMalloc(&p, want) != cudaSuccess) {
                cudaGetLastError();
                return -1;
            }
        }
        c->dev = (unsigned char *)p;
        c->dev_bytes = want;
        c->alloc_calls++;
        c->fs_growths++;
        if (c->warm) c->steady_alloc_calls++;
    }
    if (host_bytes > c->host_bytes) {
        if (c->host) {
            cudaStreamSynchronize(c->s);
            cudaFreeHost(c->host);
            c->host = nullptr;
            c->host_bytes = 0;
        }
        size_t want = host_bytes + host_bytes / 4;
        void *p = nullptr;
        if (cudaHostAlloc(&p, want, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return -1;
        }
        c->host = (unsigned char *)p;
        c->host_bytes = want;
        c->alloc_calls++;
        c->fs_growths++;
        if (c->warm) c->steady_alloc_calls++;
    }
    return 0;
}

int rc_finish(RcCtx *c)
{
    cudaEventRecord(c->ev_done, c->s);
    cudaError_t e = cudaEventSynchronize(c->ev_done);
    cudaError_t l = cudaGetLastError();
    return (e == cudaSuccess && l == cudaSuccess) ? 0 : -1;
}

__global__ void rc_cast_kernel(const float *__restrict__ src, double *__restrict__ dst, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (double)src[i];
}

int rc_ensure_f64(RcCtx *c)
{
    if (c->d_cols64 && c->d_y64) return 0;
    const size_t total = (size_t)c->npad * (size_t)c->v;
    if (!c->d_cols64) {
        if (cudaMalloc((void **)&c->d_cols64, sizeof(double) * (total ? total : 1)) != cudaSuccess) {
            cudaGetLastError();
            c->d_cols64 = nullptr;
            return -1;
        }
        c->alloc_calls++;
        if (total)
            c->launches += 1;
            rc_cast_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c->s>>>(c->d_cols, c->d_cols64,
                                                                             (long long)total);
    }
    if (!c->d_y64) {
        if (cudaMalloc((void **)&c->d_y64, sizeof(double) * c->npad) != cudaSuccess) {
            cudaGetLastError();
            c->d_y64 = nullptr;
            return -1;
        }
        c->alloc_calls++;
        c->launches += 1;
        rc_cast_kernel<<<(c->npad + 255) / 256, 256, 0, c->s>>>(c->d_y, c->d_y64, c->npad);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* Upload `n` host values into a zero-padded device vector of npad entries. */
template <typename TT>
static int upload_padded(RcCtx *c, TT **dst, const TT *src, int n, int npad)
{
    if (!*dst) {
        if (cudaMalloc((void **)dst, sizeof(TT) * (size_t)npad) != cudaSuccess) {
            cudaGetLastError();
            *dst = nullptr;
            return -1;
        }
        c->alloc_calls++;
    }
    if (cudaMemsetAsync(*dst, 0, sizeof(TT) * (size_t)npad, c->s) != cudaSuccess) return -1;
    if (n > 0 && cudaMemcpyAsync(*dst, src, sizeof(TT) * (size_t)n, cudaMemcpyHostToDevice, c->s) !=
                     cudaSuccess)
        return -1;
    return cudaStreamSynchronize(c->s) == cudaSuccess ? 0 : -1;
}

template <typename TT>
static int upload_cols(RcCtx *c, TT **dst, const TT *src)
{
    const size_t total = (size_t)c->npad * (size_t)c->v;
    if (!*dst) {
        if (cudaMalloc((void **)dst, sizeof(TT) * (total ? total : 1)) != cudaSuccess) {
            cudaGetLastError();
            *dst = nullptr;
            return -1;
        }
        c->alloc_calls++;
    }
    if (total) cudaMemsetAsync(*dst, 0, sizeof(TT) * total, c->s);
    for (int k = 0; k < c->v && c->n > 0; ++k) {
        cudaMemcpyAsync(*dst + (size_t)k * c->npad, src + (size_t)k * c->n, sizeof(TT) * c->n,
                        cudaMemcpyHostToDevice, c->s);
    }
    return cudaStreamSynchronize(c->s) == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : -1;
}

static void free_ptr(void *p)
{
    if (p) cudaFree(p);
}

extern "C" {

void *rc_create(const float *cols, int n, int v, const float *y)
{
    if (n < 0 || v < 0 || (n > 0 && (!y || (v > 0 && !cols)))) return nullptr;
    RcCtx *c = new (std::nothrow) RcCtx();
    if (!c) return nullptr;
    c->n = n;
    c->v = v;
    c->npad = ((n + RC_ROW_PAD - 1) / RC_ROW_PAD) * RC_ROW_PAD;
    if (c->npad == 0) c->npad = RC_ROW_PAD;
    c->async_copy = 1;
    const char *force_sync = getenv("RCSR_GPU_SYNC");
    if (force_sync && force_sync[0] && strcmp(force_sync, "0") != 0 &&
        strcmp(force_sync, "false") != 0 && strcmp(force_sync, "off") != 0) {
        c->async_copy = 0;
        snprintf(c->sync_reason, sizeof(c->sync_reason),
                 "RCSR_GPU_SYNC requests the synchronous copy path");
    }
    if (cudaGetDevice(&c->device) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return nullptr;
    }
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
    if (c->sm_count <= 0) c->sm_count = 1;
    if (cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->t0) != cudaSuccess || cudaEventCreate(&c->t1) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&c->sp[0]) != cudaSuccess || cudaEventCreate(&c->sp[1]) != cudaSuccess ||
        cudaEventCreate(&c->sp[2]) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return nullptr;
    }
    if (upload_cols<float>(c, &c->d_cols, cols) != 0 ||
        upload_padded<float>(c, &c->d_y, y, n, c->npad) != 0) {
        rc_destroy(c);
        return nullptr;
    }
    /* Cached target moments of the resident f32 target (eval.cu:3172-3186). */
    if (n > 0) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += (double)y[i];
        c->ybar = s / (double)n;
        double ss = 0.0;
        for (int i = 0; i < n; ++i) {
            const double d = (double)y[i] - c->ybar;
            ss += d * d;
        }
        c->syy = ss;
    }
    return c;
}

void rc_destroy(void *ctx)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c) return;
    if (c->s) cudaStreamSynchronize(c->s);
    free_ptr(c->d_cols);
    free_ptr(c->d_y);
    free_ptr(c->d_cols64);
    free_ptr(c->d_y64);
    free_ptr(c->d_w64);
    free_ptr(c->d_tsign);
    free_ptr(c->d_tsign64);
    free_ptr(c->d_rank_b);
    free_ptr(c->d_pool[0]);
    free_ptr(c->d_pool[1]);
    free_ptr(c->dev);
    if (c->host) cudaFreeHost(c->host);
    if (c->fit_graph) cudaGraphExecDestroy(c->fit_graph);
    if (c->t0) cudaEventDestroy(c->t0);
    if (c->t1) cudaEventDestroy(c->t1);
    if (c->ev_done) cudaEventDestroy(c->ev_done);
    for (int i = 0; i < 3; ++i)
        if (c->sp[i]) cudaEventDestroy(c->sp[i]);
    if (c->s) cudaStreamDestroy(c->s);
    delete c;
}

int rc_set_fit_data(void *ctx, const double *cols, const double *y, const double *w)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || (!cols && c->v > 0 && c->n > 0) || !y) return -1;
    /* New exact rows invalidate the cached target ranks (eval.cu:3890-3895). */
    c->rank_ready = 0;
    if (upload_cols<double>(c, &c->d_cols64, cols) != 0) return -1;
    if (upload_padded<double>(c, &c->d_y64, y, c->n, c->npad) != 0) return -1;
    if (w) {
        if (upload_padded<double>(c, &c->d_w64, w, c->n, c->npad) != 0) return -1;
    } else if (c->d_w64) {
        cudaFree(c->d_w64);
        c->d_w64 = nullptr;
    }
    c->fit_data_exact = 1;
    return 0;
}

int rc_set_score_weights(void *ctx, const double *w)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c) return -1;
    if (!w) {
        if (c->d_w64) cudaFree(c->d_w64);
        c->d_w64 = nullptr;
        return 0;
    }
    return upload_padded<double>(c, &c->d_w64, w, c->n, c->npad);
}

int rc_set_fit_sign(void *ctx, const double *sign)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c) return -1;
    c->has_tsign = 0;
    if (!sign) {
        free_ptr(c->d_tsign);
        free_ptr(c->d_tsign64);
        c->d_tsign = nullptr;
        c->d_tsign64 = nullptr;
        return 0;
    }
    std::vector<float> host(c->n);
    for (int i = 0; i < c->n; ++i) host[i] = (float)sign[i];
    if (upload_padded<double>(c, &c->d_tsign64, sign, c->n, c->npad) != 0) return -1;
    if (upload_padded<float>(c, &c->d_tsign, host.data(), c->n, c->npad) != 0) return -1;
    c->has_tsign = 1;
    return 0;
}

void rc_stats_begin(void *ctx)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c) return;
    memset(&c->stats, 0, sizeof(c->stats));
    c->batch_start_ms = rc_now_ms();
}

int rc_last_stats(void *ctx, RcStats *out)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !out) return -1;
    *out = c->stats;
    return 0;
}

int rc_arena_report(void *ctx, RcArenaReport *out)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c || !out) return -1;
    memset(out, 0, sizeof(*out));
    out->async_copy = c->async_copy;
    snprintf(out->reason, sizeof(out->reason), "%s", c->sync_reason);
    out->pinned_bytes = c->host_bytes;
    out->alloc_calls = c->alloc_calls;
    out->steady_alloc_calls = c->steady_alloc_calls;
    out->overlapped_uploads = 0;
    out->batches = c->batches;
    out->fs_alloc_calls = c->alloc_calls;
    out->fs_growths = c->fs_growths;
    out->fs_steady_alloc_calls = c->steady_alloc_calls;
    out->fs_batches = c->batches;
    out->fs_dev_bytes = c->dev_bytes;
    out->fs_pinned_bytes = c->host_bytes;
    return 0;
}

int rc_arena_force_sync(void *ctx, int sync)
{
    RcCtx *c = (RcCtx *)ctx;
    if (!c) return -1;
    int previous = c->async_copy;
    if (sync) {
        c->async_copy = 0;
        snprintf(c->sync_reason, sizeof(c->sync_reason), "caller forced the synchronous copy path");
    } else {
        c->async_copy = 1;
        c->sync_reason[0] = '\0';
    }
    return previous;
}

int rc_unified(void) { return 0; }

const char *rc_device_name(void)
{
    static char name[256];
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, 0) != cudaSuccess) {
        cudaGetLastError();
        return "unknown";
    }
    snprintf(name, sizeof(name), "%s (sm_%d%d, %d SMs, %d MB)", p.name, p.major, p.minor,
             p.multiProcessorCount, (int)(p.totalGlobalMem / (1024 * 1024)));
    return name;
}

int rc_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return n;
}

}  // extern "C"
