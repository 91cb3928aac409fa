// amj_bucket_build_static: the bucket-CSR build of amj_bucket_build for
// callers that cannot allocate device memory.
//
// Some hosts of this library may not call cudaMalloc at all: a plugin living
// in a query engine that owns every device byte through its own pool and
// accounts for it, or a real-time loop that may not block on the driver's
// allocator (cudaMalloc can synchronise the device and take milliseconds).
// For them this entry point works entirely in a fixed scratch area compiled
// into the library (a file-scope __device__ array), plus the input and
// output buffers the caller passes in.  It calls no cudaMalloc, cudaFree,
// cudaMallocAsync or any other allocating routine.
//
// Limits and behaviour:
//  - at most AMJ_BUCKET_STATIC_MAX_KEYS keys and AMJ_BUCKET_STATIC_MAX_BUCKETS
//    buckets per call; larger requests fail with AMJ_EINVAL;
//  - the scratch area (about 16.3 MB) is resident on every device that loads
//    the library, until the process exits;
//  - all calls share that one area: calls whose work overlaps on the GPU (two
//    host threads, or two streams, at once) race and corrupt each other's
//    results; serialise them;
//  - the first call on a device looks up the area's device address (a
//    driver query, no allocation); make that first call before any stream
//    capture begins;
//  - the call synchronises `stream` before it returns.
#include "hash_build_kernels.cuh"
#include "primitives_kernels.cuh"

#include <mutex>

namespace amj {
namespace {

constexpr uint64_t kMaxKeys = AMJ_BUCKET_STATIC_MAX_KEYS;
constexpr uint64_t kMaxBuckets = AMJ_BUCKET_STATIC_MAX_BUCKETS;
constexpr uint64_t kMaxTiles = (kMaxKeys + RS_TILE - 1) / RS_TILE;                 // radix-sort tiles
constexpr uint64_t kCountsEntries = 256 * kMaxTiles;                                // digit x tile histogram
constexpr uint64_t kPartials = ((kMaxBuckets + 1 > kCountsEntries ? kMaxBuckets + 1 : kCountsEntries) +
                                SCAN_TILE - 1) / SCAN_TILE;                         // scan tile sums
constexpr size_t kItemsOff = 0;
constexpr size_t kItemsBytes = kMaxKeys * sizeof(uint64_t);
constexpr size_t kCountsOff = 2 * kItemsBytes;
constexpr size_t kPartialOff = kCountsOff + kCountsEntries * sizeof(uint32_t);
constexpr size_t kScratchBytes = kPartialOff + ((kPartials + 63) / 64) * 64 * sizeof(uint32_t);

// The scratch area.  In host code its name only stands for the symbol: the
// device address comes from cudaGetSymbolAddress, per device.
static __device__ __align__(256) unsigned char g_bucket_scratch[kScratchBytes];

std::mutex g_setup_mu;
void *g_scratch_addr[64] = {};

int scratch_for_current_device(void **out) {
    int dev = 0;
    AMJ_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(AMJ_EINVAL, "bucket_build_static: device index beyond 63");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_bucket_scratch);
        if (e != cudaSuccess || !p) return cuda_fail(e == cudaSuccess ? cudaErrorInvalidSymbol : e,
                                                      "bucket_build_static: cudaGetSymbolAddress");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return AMJ_OK;
}

unsigned grid_for_n(uint64_t n) {
    uint64_t g = (n + 255) / 256;
    if (g > 4096) g = 4096;
    return (unsigned)(g ? g : 1);
}

// Exclusive scan of n <= SCAN_TILE * SCAN_TILE values with one level of tile
// sums held in `partial` (no allocation).
int scan_u32_fixed(cudaStream_t st, const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *partial) {
    if (n == 0) return AMJ_OK;
    const uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles > SCAN_TILE || tiles > kPartials) return fail(AMJ_EINVAL, "bucket_build_static: scan too large");
    if (tiles == 1) {
        scan_tiles_kernel<uint32_t><<<1, SCAN_THREADS, 0, st>>>(in, out, n, nullptr, nullptr);
        AMJ_CUDA_TRY(cudaGetLastError());
        return AMJ_OK;
    }
    scan_reduce_kernel<uint32_t><<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, n, partial);
    scan_tiles_kernel<uint32_t><<<1, SCAN_THREADS, 0, st>>>(partial, partial, tiles, nullptr, nullptr);
    scan_tiles_kernel<uint32_t><<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, out, n, partial, nullptr);
    AMJ_CUDA_TRY(cudaGetLastError());
    return AMJ_OK;
}

}  // namespace
}  // namespace amj

using namespace amj;

extern "C" int amj_bucket_build_static(const int32_t *d_keys, uint64_t n, uint64_t buckets, int32_t *d_hash_keys,
                                       uint32_t *d_idx_in_origin, uint32_t *d_buc_ptrs, void *stream) {
    if ((n && (!d_keys || !d_hash_keys || !d_idx_in_origin)) || !d_buc_ptrs)
        return fail(AMJ_EINVAL, "bucket_build_static: null argument");
    if (buckets == 0 || (buckets & (buckets - 1)))
        return fail(AMJ_EINVAL, "bucket_build_static: buckets must be a power of two");
    if (n > kMaxKeys)
        return fail(AMJ_EINVAL, "bucket_build_static: " + std::to_string(n) + " keys exceed the fixed scratch limit of " +
                                    std::to_string(kMaxKeys) + " (use amj_bucket_build)");
    if (buckets > kMaxBuckets)
        return fail(AMJ_EINVAL, "bucket_build_static: " + std::to_string(buckets) +
                                    " buckets exceed the fixed scratch limit of " + std::to_string(kMaxBuckets));
    void *base = nullptr;
    AMJ_TRY(scratch_for_current_device(&base));
    cudaStream_t st = (cudaStream_t)stream;
    unsigned char *scr = (unsigned char *)base;
    uint64_t *items_a = (uint64_t *)(scr + kItemsOff);
    uint64_t *items_b = (uint64_t *)(scr + kItemsOff + kItemsBytes);
    uint32_t *counts = (uint32_t *)(scr + kCountsOff);
    uint32_t *partial = (uint32_t *)(scr + kPartialOff);
    const uint32_t mask = (uint32_t)(buckets - 1);

    // bucket counts start at zero
    AMJ_CUDA_TRY(cudaMemsetAsync(d_buc_ptrs, 0, (buckets + 1) * sizeof(uint32_t), st));
    if (n) {
        pack_key_rowid_kernel<<<grid_for_n(n), 256, 0, st>>>(d_keys, n, items_a);
        AMJ_CUDA_TRY(cudaGetLastError());
        // stable LSD radix sort of (row id, key) items by the low log2(buckets) key bits
        const int nbits = log2_exact(buckets);
        uint64_t *src = items_a, *dst = items_b;
        if (nbits > 0) {
            const int passes = (nbits + 7) / 8;
            const int width = (nbits + passes - 1) / passes;
            const uint32_t nblocks = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
            for (int p = 0; p < passes; p++) {
                const int shift = p * width;
                const int bits = (nbits - shift) < width ? (nbits - shift) : width;
                rs_upsweep_kernel<SK_LOW32><<<nblocks, RS_THREADS, 0, st>>>(src, (uint32_t)n, shift, bits, counts,
                                                                            nblocks);
                AMJ_CUDA_TRY(cudaGetLastError());
                AMJ_TRY(scan_u32_fixed(st, counts, counts, (uint64_t)(1u << bits) * nblocks, partial));
                rs_downsweep_kernel<SK_LOW32><<<nblocks, RS_THREADS, 0, st>>>(src, dst, (uint32_t)n, shift, bits,
                                                                              counts, nblocks);
                AMJ_CUDA_TRY(cudaGetLastError());
                uint64_t *t = src;
                src = dst;
                dst = t;
            }
        }
        unpack_pairs_kernel<<<grid_for_n(n), 256, 0, st>>>(src, n, d_hash_keys, (int32_t *)d_idx_in_origin);
        bucket_hist_sorted_kernel<<<grid_for_n(n), 256, 0, st>>>(src, n, KEY_SINGLE, mask, d_buc_ptrs);
        AMJ_CUDA_TRY(cudaGetLastError());
    }
    AMJ_TRY(scan_u32_fixed(st, d_buc_ptrs, d_buc_ptrs, buckets + 1, partial));
    AMJ_CUDA_TRY(cudaStreamSynchronize(st));
    return AMJ_OK;
}
