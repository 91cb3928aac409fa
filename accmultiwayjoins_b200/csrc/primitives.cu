// Device primitives written for sm_100a: exclusive prefix sums and a stable
// LSD radix sort of 64-bit items.  They replace the CUB / Thrust calls of the
// reference (CUBScanExclusive common-utils/cuda/primitives.cuh:285,
// CUBSortPairsInPlace :476, thrust::sort over zip iterators
// LFTJ-GPU/multi_partitioning.cuh:174-193).
//
// Scan: reduce-then-scan over 4096-element tiles (1024 threads x 4 items),
// recursing on the tile sums.  No inter-block waiting.
//
// Radix sort: per pass an up-sweep (per-tile digit histogram, digit-major),
// a scan of the histogram, and a down-sweep that ranks each item stably
// inside its tile with warp ballots, stages the tile in shared memory in
// digit order and writes each digit run contiguously (coalesced).
#include "primitives_kernels.cuh"

namespace amj {

template <typename T>
static int scan_exclusive_impl(amj_ctx *ctx, const T *in, T *out, uint64_t n, T *d_total) {
    if (n == 0) {
        if (d_total) AMJ_CUDA_TRY(cudaMemsetAsync(d_total, 0, sizeof(T), ctx->stream));
        return AMJ_OK;
    }
    const uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles > 0x7fffffffull) return fail(AMJ_EINVAL, "scan: input too large");
    if (tiles == 1) {
        note_launch(ctx);
        scan_tiles_kernel<T><<<1, SCAN_THREADS, 0, ctx->stream>>>(in, out, n, nullptr, d_total);
        AMJ_CUDA_TRY(cudaGetLastError());
        return AMJ_OK;
    }
    DBuf<T> partial;
    AMJ_TRY(partial.alloc(ctx, tiles));
    note_launch(ctx);
    scan_reduce_kernel<T><<<(unsigned)tiles, SCAN_THREADS, 0, ctx->stream>>>(in, n, partial.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_TRY(scan_exclusive_impl<T>(ctx, partial.p, partial.p, tiles, nullptr));
    note_launch(ctx);
    scan_tiles_kernel<T><<<(unsigned)tiles, SCAN_THREADS, 0, ctx->stream>>>(in, out, n, partial.p, d_total);
    AMJ_CUDA_TRY(cudaGetLastError());
    return AMJ_OK;
}

int scan_exclusive_u32(amj_ctx *ctx, const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *d_total) {
    return scan_exclusive_impl<uint32_t>(ctx, in, out, n, d_total);
}
int scan_exclusive_u64(amj_ctx *ctx, const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *d_total) {
    return scan_exclusive_impl<uint64_t>(ctx, in, out, n, d_total);
}

template <int KK>
static int radix_sort_impl(amj_ctx *ctx, uint64_t *d_a, uint64_t *d_b, uint64_t n, int lo_bit, int hi_bit,
                           uint64_t **result) {
    *result = d_a;
    const int nbits = hi_bit - lo_bit;
    if (n <= 1 || nbits <= 0) return AMJ_OK;
    if (n > 0xffffffffull - RS_TILE) return fail(AMJ_EINVAL, "radix sort: more than 2^32 items");
    if (lo_bit < 0 || hi_bit > 64) return fail(AMJ_EINVAL, "radix sort: bad bit range");
    const int passes = (nbits + 7) / 8;
    const int width = (nbits + passes - 1) / passes;
    const uint32_t nblocks = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    DBuf<uint32_t> counts;
    AMJ_TRY(counts.alloc(ctx, (size_t)256 * nblocks));
    uint64_t *src = d_a, *dst = d_b;
    for (int p = 0; p < passes; p++) {
        const int shift = lo_bit + p * width;
        const int bits = (hi_bit - shift) < width ? (hi_bit - shift) : width;
        if (bits <= 0) break;
        note_launch(ctx);
        rs_upsweep_kernel<KK><<<nblocks, RS_THREADS, 0, ctx->stream>>>(src, (uint32_t)n, shift, bits, counts.p,
                                                                       nblocks);
        AMJ_CUDA_TRY(cudaGetLastError());
        AMJ_TRY(scan_exclusive_u32(ctx, counts.p, counts.p, (uint64_t)(1u << bits) * nblocks, nullptr));
        note_launch(ctx);
        rs_downsweep_kernel<KK><<<nblocks, RS_THREADS, 0, ctx->stream>>>(src, dst, (uint32_t)n, shift, bits,
                                                                         counts.p, nblocks);
        AMJ_CUDA_TRY(cudaGetLastError());
        uint64_t *t = src;
        src = dst;
        dst = t;
    }
    *result = src;
    return AMJ_OK;
}

int radix_sort_u64(amj_ctx *ctx, uint64_t *d_a, uint64_t *d_b, uint64_t n, int key_kind, int lo_bit, int hi_bit,
                   uint64_t **result) {
    switch (key_kind) {
        case SK_IDENT: return radix_sort_impl<SK_IDENT>(ctx, d_a, d_b, n, lo_bit, hi_bit, result);
        case SK_LOW32: return radix_sort_impl<SK_LOW32>(ctx, d_a, d_b, n, lo_bit, hi_bit, result);
        case SK_PAIR_HASH: return radix_sort_impl<SK_PAIR_HASH>(ctx, d_a, d_b, n, lo_bit, hi_bit, result);
        default: return fail(AMJ_EINVAL, "radix sort: unknown key kind");
    }
}

}  // namespace amj
