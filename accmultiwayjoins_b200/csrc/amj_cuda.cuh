// CUDA-side internals of libamj: the context, stream-ordered device buffers,
// the device status block every bounded wait reports into, and warp helpers.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "amj.h"
#include "amj_checksum.h"
#include "amj_internal.h"

#define AMJ_FULL_MASK 0xffffffffu

namespace amj {

int cuda_fail(cudaError_t e, const char *what);

#define AMJ_CUDA_TRY(call)                                          \
    do {                                                            \
        cudaError_t _amj_e = (call);                                \
        if (_amj_e != cudaSuccess) return amj::cuda_fail(_amj_e, #call); \
    } while (0)

#define AMJ_TRY(call)                  \
    do {                               \
        int _amj_rc = (call);          \
        if (_amj_rc != AMJ_OK) return _amj_rc; \
    } while (0)

// Status written by kernels.  code is a positive AMJ error number (the
// negated AMJ_E* value); the first error wins.
struct DevStatus {
    unsigned int code;
    unsigned int where;
    unsigned long long info;
    unsigned long long pad;
};

enum ErrSite : unsigned int {
    SITE_NONE = 0,
    SITE_WS_IDLE = 1,      // work-sharing idle wait
    SITE_WS_SLOT = 2,      // waiting for a pushed task to become visible
    SITE_WS_QUEUE = 3,     // task queue full where a split must not be dropped
    SITE_OUT_OVERFLOW = 4, // output buffer smaller than the result
    SITE_OA_FULL = 5,      // open-addressing table full
    SITE_CUCKOO = 6,       // cuckoo eviction chain too long
    SITE_FIB = 7,          // frequent-item buffer state wait
    SITE_LFTJ_STACK = 8,   // LFTJ depth beyond the compiled bound
    SITE_TEST_WAIT = 9,    // bounded wait exercised by the self test
};

__device__ __forceinline__ void report_error(DevStatus *st, unsigned int code, unsigned int where,
                                             unsigned long long info) {
    if (atomicCAS(&st->code, 0u, code) == 0u) {
        st->where = where;
        st->info = info;
    }
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned int lanemask_lt() {
    unsigned int m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = __shfl_up_sync(AMJ_FULL_MASK, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(AMJ_FULL_MASK, v, d);
    return v;
}

__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t *p) {
    return *(const volatile uint32_t *)p;
}
__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long *p) {
    return *(const volatile unsigned long long *)p;
}

// composite hash of a 2-attribute key
__host__ __device__ __forceinline__ uint32_t hash_pair(int32_t a, int32_t b) {
    return (uint32_t)(amj_mix64(((uint64_t)(uint32_t)a << 32) | (uint32_t)b) >> 32);
}
// single-key hash for open addressing / cuckoo tables (murmur3 finaliser,
// the hash the reference's linear-probing table uses, MHJ-GPU/common_kernels.cuh:12-19)
__host__ __device__ __forceinline__ uint32_t hash_key(int32_t k) {
    uint32_t h = (uint32_t)k;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

}  // namespace amj

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
namespace amj {
struct IndexProvider;
}

struct amj_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    amj_opts opts{};
    int num_sms = 148;
    int max_smem_optin = 227 * 1024;
    size_t device_mem = 0;               // total device memory (bytes)
    size_t l2_bytes = 0;
    amj::DevStatus *d_status = nullptr;    // device status block
    amj::DevStatus *h_status = nullptr;    // pinned host mirror
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaStream_t side_stream[2] = {nullptr, nullptr};   // ooc copy / prefetch streams
    unsigned long long launches = 0;                     // kernels launched through this context
    cudaEvent_t kev[4] = {nullptr, nullptr, nullptr, nullptr};   // per-kernel timing
    amj::IndexProvider *iprov = nullptr;   // indexes kept across calls (set by the request server)
    void *c4_mtx = nullptr;                // 4-clique triangle matrices, kept across calls (grow-only)
    uint64_t c4_mtx_words = 0;
    void *pinned_cache = nullptr;          // pinned host blocks of out-of-core stages, kept across calls
};

struct amj_rel {
    amj_ctx *ctx = nullptr;
    uint64_t uid = 0;                          // serial number, unique for the process's lifetime
    uint64_t n = 0;
    int ncols = 0;
    uint32_t attrs[AMJ_MAX_COLS] = {};
    int32_t *d_cols[AMJ_MAX_COLS] = {};        // device columns (owned when `owned`)
    const int32_t *h_cols[AMJ_MAX_COLS] = {};  // host columns (AMJ_MEM_HOST_STREAMED)
    int where = AMJ_MEM_DEVICE;
    bool owned = false;
};

namespace amj {

inline void note_launch(amj_ctx *ctx) { ctx->launches++; }

// Stream-ordered device allocation on the context stream.
int dev_alloc(amj_ctx *ctx, void **p, size_t bytes);
void dev_free(amj_ctx *ctx, void *p);
// Free the pinned host blocks the context keeps for out-of-core stages.
void pinned_cache_release(amj_ctx *ctx);

template <typename T>
struct DBuf {
    amj_ctx *ctx = nullptr;
    T *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    DBuf(DBuf &&o) noexcept : ctx(o.ctx), p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DBuf &operator=(DBuf &&o) noexcept {
        if (this != &o) {
            release();
            ctx = o.ctx; p = o.p; n = o.n;
            o.p = nullptr; o.n = 0;
        }
        return *this;
    }
    int alloc(amj_ctx *c, size_t count) {
        release();
        ctx = c;
        n = count;
        if (count == 0) return AMJ_OK;
        return dev_alloc(c, (void **)&p, count * sizeof(T));
    }
    void release() {
        if (p && ctx) dev_free(ctx, p);
        p = nullptr;
        n = 0;
    }
    T *detach() { T *q = p; p = nullptr; n = 0; return q; }
    ~DBuf() { release(); }
};

// Clear the device status block (enqueued on the context stream).
int status_reset(amj_ctx *ctx);
// Synchronise the context stream, then convert a device-side error into a
// status code and message.
int status_check(amj_ctx *ctx, const char *what);

// ---- primitives (primitives.cu) ----
// exclusive prefix sum; out may alias in; *d_total (device, optional) receives the sum
int scan_exclusive_u32(amj_ctx *ctx, const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *d_total);
int scan_exclusive_u64(amj_ctx *ctx, const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *d_total);

// sort-key functions for the radix sort
enum SortKeyKind : int {
    SK_IDENT = 0,      // the item itself
    SK_LOW32 = 1,      // low 32 bits of the item (single-key bucket: key in the low word)
    SK_PAIR_HASH = 2,  // hash_pair(low word, high word): composite-key bucket
};
// LSD radix sort of n 64-bit items by bits [lo_bit, hi_bit) of key(item);
// stable.  Ping-pongs between d_a and d_b; *result points at the sorted copy.
int radix_sort_u64(amj_ctx *ctx, uint64_t *d_a, uint64_t *d_b, uint64_t n, int key_kind, int lo_bit,
                   int hi_bit, uint64_t **result);

}  // namespace amj
