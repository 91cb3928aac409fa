// Hash-index construction for AMHJ build relations.
//
// Bucket layout (reference: RadixPartitioner::splitKI,
// MHJ-GPU/Indexing/radix_partitioning.cuh:508-578, bucket = key & (B-1) with
// B = floorPow2(n) as in MHJ-GPU/QueryProcessor.cuh:86): the (c0, c1) pairs
// are packed into 64-bit items and radix sorted by the bucket bits of their
// key (stable, so rows inside a bucket stay in row order), unpacked into
// bucket-ordered columns, and the bucket offsets come from a run-length
// histogram of the sorted bucket ids plus an exclusive scan.
//
// Open addressing (reference: MHJ-GPU/Indexing/linear.cuh:12-33, murmur3,
// capacity ceilPow2(n / 0.5)): 8-byte (c0, c1) slots claimed with one 64-bit
// CAS so key and payload appear together.
//
// Bucketised cuckoo (reference: MHJ-GPU/Indexing/cuckoo_radix.cuh:25-125):
// two hash functions, 4-slot buckets that fill exactly one 32-byte sector, an
// eviction chain bounded in length; a key can appear at most 8 times.
#include "hash_build_kernels.cuh"

namespace amj {

__global__ void pack_pairs_kernel(const int32_t *__restrict__ c0, const int32_t *__restrict__ c1, uint64_t n,
                                  uint64_t *__restrict__ items) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t hi = c1 ? (uint32_t)c1[i] : 0u;
        items[i] = ((uint64_t)hi << 32) | (uint32_t)c0[i];
    }
}

__global__ void gather_col_kernel(const uint64_t *__restrict__ items, uint64_t n, const int32_t *__restrict__ src,
                                  int32_t *__restrict__ dst) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[(uint32_t)(items[i] >> 32)];
}

__global__ void fill_slots_kernel(int2 *slots, uint64_t m) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        slots[i] = make_int2(OA_EMPTY_KEY, 0);
}

__device__ __forceinline__ unsigned long long pack_slot(int32_t x, int32_t y) {
    return ((unsigned long long)(uint32_t)y << 32) | (uint32_t)x;
}

__device__ __forceinline__ uint32_t oa_hash(int32_t c0, int32_t c1, int key_mode) {
    return key_mode == KEY_PAIR ? hash_pair(c0, c1) : hash_key(c0);
}

__global__ void oa_insert_kernel(const int32_t *__restrict__ c0, const int32_t *__restrict__ c1, uint64_t n,
                                 int key_mode, uint32_t mask, int2 *slots, DevStatus *st) {
    const unsigned long long empty = pack_slot(OA_EMPTY_KEY, 0);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const int32_t x = c0[i], y = c1 ? c1[i] : 0;
        if (x == OA_EMPTY_KEY) {
            report_error(st, (unsigned)-AMJ_EINVAL, SITE_OA_FULL, i);
            continue;
        }
        const unsigned long long want = pack_slot(x, y);
        uint32_t s = oa_hash(x, y, key_mode) & mask;
        bool done = false;
        for (uint64_t probe = 0; probe <= mask; probe++) {
            unsigned long long prev = atomicCAS((unsigned long long *)&slots[s], empty, want);
            if (prev == empty) {
                done = true;
                break;
            }
            s = (s + 1) & mask;
        }
        if (!done) report_error(st, (unsigned)-AMJ_EOVERFLOW, SITE_OA_FULL, i);
    }
}

__device__ __forceinline__ uint32_t cuckoo_h1(int32_t c0, int32_t c1, int key_mode) {
    return oa_hash(c0, c1, key_mode);
}
__device__ __forceinline__ uint32_t cuckoo_h2(int32_t c0, int32_t c1, int key_mode) {
    uint32_t h = oa_hash(c0, c1, key_mode);
    return hash_key((int32_t)(h ^ 0x5bd1e995u)) ^ 0x9e3779b9u;
}

__global__ void cuckoo_insert_kernel(const int32_t *__restrict__ c0, const int32_t *__restrict__ c1, uint64_t n,
                                     int key_mode, uint32_t bmask, int2 *slots, int max_evict, DevStatus *st) {
    const unsigned long long empty = pack_slot(OA_EMPTY_KEY, 0);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        int32_t x = c0[i], y = c1 ? c1[i] : 0;
        if (x == OA_EMPTY_KEY) {
            report_error(st, (unsigned)-AMJ_EINVAL, SITE_CUCKOO, i);
            continue;
        }
        unsigned long long cur = pack_slot(x, y);
        uint32_t b = cuckoo_h1(x, y, key_mode) & bmask;
        bool placed = false;
        for (int it = 0; it < max_evict && !placed; it++) {
            for (int s = 0; s < CUCKOO_SLOTS; s++) {
                unsigned long long prev =
                    atomicCAS((unsigned long long *)&slots[(uint64_t)b * CUCKOO_SLOTS + s], empty, cur);
                if (prev == empty) {
                    placed = true;
                    break;
                }
            }
            if (placed) break;
            // evict a slot chosen by the step number and move the victim to its other bucket
            const int victim = (int)((i + it) & (CUCKOO_SLOTS - 1));
            unsigned long long old =
                atomicExch((unsigned long long *)&slots[(uint64_t)b * CUCKOO_SLOTS + victim], cur);
            if (old == empty) {
                placed = true;
                break;
            }
            cur = old;
            const int32_t ox = (int32_t)(uint32_t)old, oy = (int32_t)(uint32_t)(old >> 32);
            const uint32_t b1 = cuckoo_h1(ox, oy, key_mode) & bmask, b2 = cuckoo_h2(ox, oy, key_mode) & bmask;
            b = (b == b1) ? b2 : b1;
        }
        if (!placed) report_error(st, (unsigned)-AMJ_EOVERFLOW, SITE_CUCKOO, i);
    }
}

static unsigned grid_for(amj_ctx *ctx, uint64_t n, int threads = 256) {
    uint64_t g = (n + threads - 1) / threads;
    uint64_t cap = (uint64_t)ctx->num_sms * 16;
    if (g > cap) g = cap;
    if (g == 0) g = 1;
    return (unsigned)g;
}

// ---- counting build (the operator's indexes up to BUCKET_COUNT_MAX rows) ----
// One count pass over the rows' buckets, a scan, and one scatter pass that
// claims each row's slot with an atomic on its bucket's cursor: three
// kernels instead of the radix sort's passes, which are launch-bound at
// these sizes.  The lanes of a warp that fall in one bucket share one atomic
// (a hot key costs one atomic per warp, not per row).  Rows keep no order
// inside a bucket, as in the reference's build (shared-memory atomics); every
// probe path reads a bucket as a set.
constexpr uint64_t BUCKET_COUNT_MAX = 1ull << 23;

struct BucketCols {
    const int32_t *in[4];
    int32_t *out[4];
    int ncols;
    int key_mode;
    uint32_t mask;
};

__device__ __forceinline__ uint32_t row_bucket(const BucketCols &C, uint64_t i) {
    const uint32_t k = C.key_mode == KEY_PAIR ? hash_pair(C.in[0][i], C.in[1][i]) : (uint32_t)C.in[0][i];
    return k & C.mask;
}

__global__ void bucket_count_kernel(const BucketCols C, uint64_t n, uint32_t *__restrict__ counts) {
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        const uint64_t i = base + lane;
        const bool valid = i < n;
        const uint32_t b = valid ? row_bucket(C, i) : 0xffffffffu;
        const unsigned peers = __match_any_sync(AMJ_FULL_MASK, b);
        if (valid && (peers & lanemask_lt()) == 0) atomicAdd(&counts[b], (uint32_t)__popc(peers));
    }
}

__global__ void bucket_scatter_kernel(const BucketCols C, uint64_t n, uint32_t *__restrict__ cursor) {
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        const uint64_t i = base + lane;
        const bool valid = i < n;
        const uint32_t b = valid ? row_bucket(C, i) : 0xffffffffu;
        const unsigned peers = __match_any_sync(AMJ_FULL_MASK, b);
        const int leader = __ffs(peers) - 1;
        uint32_t at = 0;
        if (valid && lane == leader) at = atomicAdd(&cursor[b], (uint32_t)__popc(peers));
        at = __shfl_sync(AMJ_FULL_MASK, at, leader);
        if (valid) {
            const uint32_t pos = at + __popc(peers & lanemask_lt());
            for (int c = 0; c < C.ncols; c++) C.out[c][pos] = C.in[c][i];
        }
    }
}

static int build_bucket_counting(amj_ctx *ctx, const int32_t *const *d_cols, int ncols, uint64_t n, int key_mode,
                                 uint64_t B, HashIndex *out) {
    BucketCols C{};
    for (int c = 0; c < ncols; c++) {
        C.in[c] = d_cols[c];
        C.out[c] = out->cols[c].p;
    }
    C.ncols = ncols;
    C.key_mode = key_mode;
    C.mask = out->mask;
    AMJ_CUDA_TRY(cudaMemsetAsync(out->buc_ptrs.p, 0, (B + 1) * sizeof(uint32_t), ctx->stream));
    note_launch(ctx);
    bucket_count_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(C, n, out->buc_ptrs.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_TRY(scan_exclusive_u32(ctx, out->buc_ptrs.p, out->buc_ptrs.p, B + 1, nullptr));
    DBuf<uint32_t> cursor;
    AMJ_TRY(cursor.alloc(ctx, B));
    AMJ_CUDA_TRY(cudaMemcpyAsync(cursor.p, out->buc_ptrs.p, B * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                                 ctx->stream));
    note_launch(ctx);
    bucket_scatter_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(C, n, cursor.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    return AMJ_OK;
}

static int build_bucket(amj_ctx *ctx, const int32_t *const *d_cols, int ncols, uint64_t n, int key_mode,
                        HashIndex *out) {
    const uint64_t B = n ? floor_pow2(n) : 1;
    if (B > (1ull << 31)) return fail(AMJ_EINVAL, "bucket index: too many rows");
    const int bits = log2_exact(B);
    out->mask = (uint32_t)(B - 1);
    AMJ_TRY(out->buc_ptrs.alloc(ctx, B + 1));
    for (int c = 0; c < ncols; c++) AMJ_TRY(out->cols[c].alloc(ctx, n ? n : 1));
    if (n == 0) {
        AMJ_CUDA_TRY(cudaMemsetAsync(out->buc_ptrs.p, 0, (B + 1) * sizeof(uint32_t), ctx->stream));
        return AMJ_OK;
    }
    if (n <= BUCKET_COUNT_MAX) return build_bucket_counting(ctx, d_cols, ncols, n, key_mode, B, out);
    DBuf<uint64_t> a, b;
    AMJ_TRY(a.alloc(ctx, n));
    AMJ_TRY(b.alloc(ctx, n));
    const bool pairs = ncols <= 2;
    if (pairs) {
        note_launch(ctx);
        pack_pairs_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(d_cols[0], ncols > 1 ? d_cols[1] : nullptr, n,
                                                                      a.p);
    } else {
        if (key_mode != KEY_SINGLE) return fail(AMJ_EUNSUPPORTED, "bucket index: pair key needs a 2-column relation");
        note_launch(ctx);
        pack_key_rowid_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(d_cols[0], n, a.p);
    }
    AMJ_CUDA_TRY(cudaGetLastError());
    uint64_t *sorted = nullptr;
    AMJ_TRY(radix_sort_u64(ctx, a.p, b.p, n, key_mode == KEY_PAIR ? SK_PAIR_HASH : SK_LOW32, 0, bits, &sorted));
    if (pairs) {
        note_launch(ctx);
        unpack_pairs_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sorted, n, out->cols[0].p,
                                                                        ncols > 1 ? out->cols[1].p : nullptr);
    } else {
        note_launch(ctx);
        unpack_pairs_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sorted, n, out->cols[0].p, nullptr);
        for (int c = 1; c < ncols; c++) {
            note_launch(ctx);
            gather_col_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sorted, n, d_cols[c], out->cols[c].p);
        }
    }
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_CUDA_TRY(cudaMemsetAsync(out->buc_ptrs.p, 0, (B + 1) * sizeof(uint32_t), ctx->stream));
    note_launch(ctx);
    bucket_hist_sorted_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(
        sorted, n, pairs ? key_mode : KEY_SINGLE, out->mask, out->buc_ptrs.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_TRY(scan_exclusive_u32(ctx, out->buc_ptrs.p, out->buc_ptrs.p, B + 1, nullptr));
    return AMJ_OK;
}

int build_hash_index(amj_ctx *ctx, const int32_t *const *d_cols, int ncols, uint64_t n, int layout, int key_mode,
                     float load_factor, HashIndex *out) {
    if (ncols <= 0 || ncols > 4) return fail(AMJ_EUNSUPPORTED, "hash index: build relations have 1..4 columns");
    if (key_mode == KEY_PAIR && ncols != 2) return fail(AMJ_EUNSUPPORTED, "hash index: pair key needs 2 columns");
    if (n >= (1ull << 32)) return fail(AMJ_EUNSUPPORTED, "hash index: build relation has 2^32 or more rows");
    out->layout = layout;
    out->key_mode = key_mode;
    out->n = n;
    out->ncols = ncols;
    if (layout == AMJ_LAYOUT_BUCKET) return build_bucket(ctx, d_cols, ncols, n, key_mode, out);
    if (ncols > 2) return fail(AMJ_EUNSUPPORTED, "open addressing / cuckoo: build relations have 1..2 columns");
    if (!(load_factor > 0.f && load_factor < 1.f)) load_factor = 0.5f;
    AMJ_TRY(status_reset(ctx));
    if (layout == AMJ_LAYOUT_OPEN_ADDR) {
        uint64_t cap = ceil_pow2((uint64_t)((double)n / load_factor) + 1);
        if (cap < 32) cap = 32;
        if (cap > (1ull << 31)) return fail(AMJ_EINVAL, "open addressing: capacity too large");
        out->mask = (uint32_t)(cap - 1);
        AMJ_TRY(out->slots.alloc(ctx, cap));
        note_launch(ctx);
        fill_slots_kernel<<<grid_for(ctx, cap), 256, 0, ctx->stream>>>(out->slots.p, cap);
        note_launch(ctx);
        oa_insert_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(d_cols[0], ncols > 1 ? d_cols[1] : nullptr, n,
                                                                     key_mode, out->mask, out->slots.p, ctx->d_status);
        AMJ_CUDA_TRY(cudaGetLastError());
        return status_check(ctx, "open-addressing build");
    }
    if (layout == AMJ_LAYOUT_CUCKOO) {
        uint64_t nb = ceil_pow2((uint64_t)((double)n / (CUCKOO_SLOTS * load_factor)) + 1);
        if (nb < 8) nb = 8;
        if (nb * CUCKOO_SLOTS > (1ull << 31)) return fail(AMJ_EINVAL, "cuckoo: capacity too large");
        out->mask = (uint32_t)(nb - 1);
        AMJ_TRY(out->slots.alloc(ctx, nb * CUCKOO_SLOTS));
        note_launch(ctx);
        fill_slots_kernel<<<grid_for(ctx, nb * CUCKOO_SLOTS), 256, 0, ctx->stream>>>(out->slots.p, nb * CUCKOO_SLOTS);
        note_launch(ctx);
        cuckoo_insert_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(
            d_cols[0], ncols > 1 ? d_cols[1] : nullptr, n, key_mode, out->mask, out->slots.p, 256, ctx->d_status);
        AMJ_CUDA_TRY(cudaGetLastError());
        return status_check(ctx, "cuckoo build");
    }
    return fail(AMJ_EINVAL, "hash index: unknown layout");
}

}  // namespace amj

using namespace amj;

extern "C" int amj_bucket_build(amj_ctx *ctx, const int32_t *d_keys, uint64_t n, uint64_t buckets,
                                int32_t *d_hash_keys, uint32_t *d_idx_in_origin, uint32_t *d_buc_ptrs) {
    if (!ctx || (n && (!d_keys || !d_hash_keys || !d_idx_in_origin)) || !d_buc_ptrs)
        return fail(AMJ_EINVAL, "bucket_build: null argument");
    if (buckets == 0 || (buckets & (buckets - 1)) || buckets > (1ull << 31))
        return fail(AMJ_EINVAL, "bucket_build: buckets must be a power of two <= 2^31");
    if (n >= (1ull << 32)) return fail(AMJ_EINVAL, "bucket_build: n must be < 2^32");
    const uint32_t mask = (uint32_t)(buckets - 1);
    AMJ_CUDA_TRY(cudaMemsetAsync(d_buc_ptrs, 0, (buckets + 1) * sizeof(uint32_t), ctx->stream));
    if (n) {
        DBuf<uint64_t> a, b;
        AMJ_TRY(a.alloc(ctx, n));
        AMJ_TRY(b.alloc(ctx, n));
        note_launch(ctx);
        pack_key_rowid_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(d_keys, n, a.p);
        AMJ_CUDA_TRY(cudaGetLastError());
        uint64_t *sorted = nullptr;
        AMJ_TRY(radix_sort_u64(ctx, a.p, b.p, n, SK_LOW32, 0, log2_exact(buckets), &sorted));
        note_launch(ctx);
        unpack_pairs_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sorted, n, d_hash_keys,
                                                                        (int32_t *)d_idx_in_origin);
        note_launch(ctx);
        bucket_hist_sorted_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sorted, n, KEY_SINGLE, mask, d_buc_ptrs);
        AMJ_CUDA_TRY(cudaGetLastError());
    }
    AMJ_TRY(scan_exclusive_u32(ctx, d_buc_ptrs, d_buc_ptrs, buckets + 1, nullptr));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return AMJ_OK;
}
