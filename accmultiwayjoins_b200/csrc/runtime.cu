// Context, device memory, status block, relations and results.
//
// The reference allocates everything with cudaMallocManaged plus prefetch and
// never frees (common-utils/cuda/CUDAStat.cuh:126-146); it exits on any CUDA
// error (common-utils/cuda/cuda_base.cuh:43-57).  Here every allocation is
// stream ordered (cudaMallocAsync on the context stream, served by the
// device's memory pool), every relation / result has an owner, and errors
// come back as status codes with a per-thread message.
#include "amj_cuda.cuh"

#include <atomic>
#include "amj_ops.cuh"

#include <cstdio>
#include <cstring>
#include <mutex>

namespace amj {

static thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    (void)cudaGetLastError();  // clear a sticky-free error so the context stays usable
    int code = (e == cudaErrorMemoryAllocation) ? AMJ_ENOMEM : AMJ_ECUDA;
    return fail(code, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

int dev_alloc(amj_ctx *ctx, void **p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) return AMJ_OK;
    cudaError_t e = cudaMallocAsync(p, bytes, ctx->stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        (void)cudaGetLastError();
        return fail(AMJ_ENOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed: " +
                                    cudaGetErrorString(e));
    }
    return AMJ_OK;
}

void dev_free(amj_ctx *ctx, void *p) {
    if (p) (void)cudaFreeAsync(p, ctx->stream);
}

int status_reset(amj_ctx *ctx) {
    AMJ_CUDA_TRY(cudaMemsetAsync(ctx->d_status, 0, sizeof(DevStatus), ctx->stream));
    return AMJ_OK;
}

static const char *site_name(unsigned w) {
    switch (w) {
        case SITE_WS_IDLE: return "work-sharing idle wait";
        case SITE_WS_SLOT: return "work-sharing task publication wait";
        case SITE_WS_QUEUE: return "work-sharing task queue";
        case SITE_OUT_OVERFLOW: return "output buffer";
        case SITE_OA_FULL: return "open-addressing table";
        case SITE_CUCKOO: return "cuckoo insertion";
        case SITE_FIB: return "frequent-item buffer";
        case SITE_LFTJ_STACK: return "LFTJ stack";
        case SITE_TEST_WAIT: return "test wait";
        default: return "kernel";
    }
}

int status_check(amj_ctx *ctx, const char *what) {
    AMJ_CUDA_TRY(cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, what);
    const DevStatus s = *ctx->h_status;
    if (s.code == 0) return AMJ_OK;
    const int code = -(int)s.code;
    std::string msg = std::string(what) + ": device reported ";
    switch (code) {
        case AMJ_ETIMEOUT: msg += "a bounded wait that ran out"; break;
        case AMJ_EOVERFLOW: msg += "an overflow"; break;
        default: msg += "error " + std::to_string(code); break;
    }
    msg += std::string(" in ") + site_name(s.where) + " (info " + std::to_string(s.info) + ")";
    return fail(code, msg);
}

// A wait on a flag that nothing sets: it must give up after limit_ns, record
// AMJ_ETIMEOUT in the status block and return, leaving the context usable.
__global__ void bounded_wait_kernel(const unsigned int *flag, unsigned long long limit_ns, DevStatus *st) {
    const unsigned long long t0 = globaltimer_ns();
    while (ld_volatile_u32(flag) == 0u) {
        if (globaltimer_ns() - t0 > limit_ns) {
            report_error(st, (unsigned)-AMJ_ETIMEOUT, SITE_TEST_WAIT, limit_ns);
            return;
        }
        __nanosleep(1000);
    }
}

}  // namespace amj

using namespace amj;

extern "C" int amj_selftest_bounded_wait(amj_ctx *ctx, uint32_t limit_ms) {
    if (!ctx || limit_ms == 0 || limit_ms > 60000) return fail(AMJ_EINVAL, "selftest_bounded_wait: bad arguments");
    DBuf<unsigned int> flag;
    AMJ_TRY(flag.alloc(ctx, 1));
    AMJ_CUDA_TRY(cudaMemsetAsync(flag.p, 0, sizeof(unsigned int), ctx->stream));
    AMJ_TRY(status_reset(ctx));
    note_launch(ctx);
    bounded_wait_kernel<<<1, 32, 0, ctx->stream>>>(flag.p, (unsigned long long)limit_ms * 1000000ull, ctx->d_status);
    AMJ_CUDA_TRY(cudaGetLastError());
    int rc = status_check(ctx, "selftest_bounded_wait");
    (void)status_reset(ctx);
    return rc;
}

extern "C" const char *amj_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *amj_version(void) { return "amj 0.1.0 (sm_100a)"; }

extern "C" int amj_ctx_create(int device, const amj_opts *opts, amj_ctx **out) {
    if (!out) return fail(AMJ_EINVAL, "ctx_create: null out");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        return fail(AMJ_ECUDA, "ctx_create: no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(AMJ_EINVAL, "ctx_create: device index out of range");
    AMJ_CUDA_TRY(cudaSetDevice(device));
    auto *c = new amj_ctx();
    c->device = device;
    if (opts) c->opts = *opts;
    if (c->opts.block_size <= 0) c->opts.block_size = 256;
    if (c->opts.load_factor <= 0.f || c->opts.load_factor >= 1.f) c->opts.load_factor = 0.5f;
    if (c->opts.task_chunk <= 0) c->opts.task_chunk = 1024;
    if (c->opts.spin_limit_ms == 0) c->opts.spin_limit_ms = 5000;
    if (c->opts.task_capacity == 0) c->opts.task_capacity = 1ull << 22;
    cudaDeviceProp prop;
    AMJ_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    c->num_sms = prop.multiProcessorCount;
    c->max_smem_optin = (int)prop.sharedMemPerBlockOptin;
    c->device_mem = prop.totalGlobalMem;
    c->l2_bytes = prop.l2CacheSize;
    int rc = AMJ_OK;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) rc = AMJ_ECUDA;
    c->own_stream = true;
    for (int i = 0; rc == AMJ_OK && i < 2; i++)
        if (cudaStreamCreateWithFlags(&c->side_stream[i], cudaStreamNonBlocking) != cudaSuccess) rc = AMJ_ECUDA;
    for (int i = 0; rc == AMJ_OK && i < 4; i++)
        if (cudaEventCreate(&c->ev[i]) != cudaSuccess || cudaEventCreate(&c->kev[i]) != cudaSuccess) rc = AMJ_ECUDA;
    if (rc == AMJ_OK && cudaMalloc((void **)&c->d_status, sizeof(DevStatus)) != cudaSuccess) rc = AMJ_ENOMEM;
    if (rc == AMJ_OK && cudaMallocHost((void **)&c->h_status, sizeof(DevStatus)) != cudaSuccess) rc = AMJ_ENOMEM;
    if (rc == AMJ_OK && cudaMemset(c->d_status, 0, sizeof(DevStatus)) != cudaSuccess) rc = AMJ_ECUDA;
    if (rc != AMJ_OK) {
        (void)cudaGetLastError();
        amj_ctx_destroy(c);
        return fail(rc, "ctx_create: failed to create streams, events or the status block");
    }
    // Keep freed blocks in the pool across calls instead of returning them
    // to the driver at every synchronisation.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        (void)cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    (void)cudaGetLastError();
    *out = c;
    return AMJ_OK;
}

extern "C" void amj_ctx_destroy(amj_ctx *c) {
    if (!c) return;
    (void)cudaSetDevice(c->device);
    if (c->stream) (void)cudaStreamSynchronize(c->stream);
    for (int i = 0; i < 4; i++) {
        if (c->ev[i]) (void)cudaEventDestroy(c->ev[i]);
        if (c->kev[i]) (void)cudaEventDestroy(c->kev[i]);
    }
    for (int i = 0; i < 2; i++)
        if (c->side_stream[i]) (void)cudaStreamDestroy(c->side_stream[i]);
    if (c->d_status) (void)cudaFree(c->d_status);
    if (c->h_status) (void)cudaFreeHost(c->h_status);
    if (c->c4_mtx) (void)cudaFree(c->c4_mtx);
    amj::pinned_cache_release(c);
    if (c->own_stream && c->stream) (void)cudaStreamDestroy(c->stream);
    (void)cudaGetLastError();
    delete c;
}

extern "C" int amj_ctx_set_stream(amj_ctx *c, void *s) {
    if (!c) return fail(AMJ_EINVAL, "ctx_set_stream: null ctx");
    AMJ_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->own_stream) (void)cudaStreamDestroy(c->stream);
    c->stream = (cudaStream_t)s;
    c->own_stream = false;
    return AMJ_OK;
}

extern "C" int amj_ctx_sync(amj_ctx *c) {
    if (!c) return fail(AMJ_EINVAL, "ctx_sync: null ctx");
    AMJ_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return AMJ_OK;
}

extern "C" int amj_ctx_launch_count(const amj_ctx *c, uint64_t *out) {
    if (!c || !out) return fail(AMJ_EINVAL, "ctx_launch_count: null argument");
    *out = c->launches;
    return AMJ_OK;
}

extern "C" int amj_ctx_trim(amj_ctx *c) {
    if (!c) return fail(AMJ_EINVAL, "ctx_trim: null ctx");
    AMJ_CUDA_TRY(cudaSetDevice(c->device));
    AMJ_CUDA_TRY(cudaStreamSynchronize(c->stream));
    amj::pinned_cache_release(c);
    if (c->c4_mtx) {
        AMJ_CUDA_TRY(cudaFree(c->c4_mtx));
        c->c4_mtx = nullptr;
        c->c4_mtx_words = 0;
    }
    return AMJ_OK;
}

extern "C" const char *amj_stat_name(int i) {
    static const char *names[12] = {"tasks_pushed", "tasks_popped", "residual_units", "rows_written_main",
                                    "rows_written_residual", "estimate", "fallbacks", "slices",
                                    "fib_keys", "fib_rows_cached", "fib_rows_served", "batch_queries"};
    return (i >= 0 && i < 12) ? names[i] : "";
}

// ---- relations ----
extern "C" int amj_rel_create(amj_ctx *ctx, uint64_t n, int ncols, const uint32_t *attrs,
                              const int32_t *const *cols, int where, amj_rel **out) {
    if (!ctx || !out || ncols <= 0 || ncols > AMJ_MAX_COLS || !attrs || (n && !cols))
        return fail(AMJ_EINVAL, "rel_create: bad arguments");
    *out = nullptr;
    for (int c = 0; c < ncols; c++) {
        if (attrs[c] >= AMJ_MAX_ATTRS) return fail(AMJ_EINVAL, "rel_create: attribute id >= AMJ_MAX_ATTRS");
        if (n && !cols[c]) return fail(AMJ_EINVAL, "rel_create: null column");
        for (int d = 0; d < c; d++)
            if (attrs[d] == attrs[c]) return fail(AMJ_EINVAL, "rel_create: repeated attribute in one relation");
    }
    static std::atomic<uint64_t> next_uid{1};
    auto *r = new amj_rel();
    r->ctx = ctx;
    r->uid = next_uid.fetch_add(1);
    r->n = n;
    r->ncols = ncols;
    r->where = where;
    for (int c = 0; c < ncols; c++) r->attrs[c] = attrs[c];
    if (where == AMJ_MEM_DEVICE) {
        for (int c = 0; c < ncols; c++) r->d_cols[c] = const_cast<int32_t *>(cols[c]);
    } else if (where == AMJ_MEM_HOST) {
        r->owned = true;
        for (int c = 0; c < ncols; c++) {
            int rc = dev_alloc(ctx, (void **)&r->d_cols[c], n * sizeof(int32_t));
            if (rc == AMJ_OK && n) {
                cudaError_t e = cudaMemcpyAsync(r->d_cols[c], cols[c], n * sizeof(int32_t), cudaMemcpyHostToDevice,
                                                ctx->stream);
                if (e != cudaSuccess) rc = cuda_fail(e, "rel_create: host to device copy");
            }
            if (rc != AMJ_OK) {
                amj_rel_release(r);
                return rc;
            }
        }
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            amj_rel_release(r);
            return cuda_fail(e, "rel_create: synchronize");
        }
    } else if (where == AMJ_MEM_HOST_STREAMED) {
        for (int c = 0; c < ncols; c++) r->h_cols[c] = cols[c];
    } else {
        delete r;
        return fail(AMJ_EINVAL, "rel_create: unknown residency");
    }
    *out = r;
    return AMJ_OK;
}

extern "C" void amj_rel_release(amj_rel *r) {
    if (!r) return;
    if (r->owned)
        for (int c = 0; c < r->ncols; c++) dev_free(r->ctx, r->d_cols[c]);
    delete r;
}

extern "C" int amj_rel_info(const amj_rel *r, uint64_t *n, int *ncols, uint32_t *attrs) {
    if (!r) return fail(AMJ_EINVAL, "rel_info: null relation");
    if (n) *n = r->n;
    if (ncols) *ncols = r->ncols;
    if (attrs)
        for (int c = 0; c < r->ncols; c++) attrs[c] = r->attrs[c];
    return AMJ_OK;
}

// ---- results ----
namespace amj {
void result_init(amj_result *res, int k) {
    std::memset(res, 0, sizeof(*res));
    res->num_attrs = k;
}
}  // namespace amj

extern "C" void amj_result_release(amj_result *res) {
    if (!res) return;
    auto *o = (ResultOwner *)res->priv;
    if (o) {
        if (o->ctx) (void)cudaSetDevice(o->ctx->device);
        for (int a = 0; a < AMJ_MAX_ATTRS; a++) {
            if (!res->cols[a]) continue;
            if (res->on_host) (void)cudaFreeHost(res->cols[a]);
            else if (o->ctx) dev_free(o->ctx, res->cols[a]);
        }
        if (o->ctx && !res->on_host) (void)cudaStreamSynchronize(o->ctx->stream);
        delete o;
    }
    for (int a = 0; a < AMJ_MAX_ATTRS; a++) res->cols[a] = nullptr;
    res->priv = nullptr;
    res->rows = 0;
}
