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
#include "amj_cuda.cuh"

namespace amj {

// ------------------------------------------------------------------ scan --
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_IPT = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_IPT;

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *wsum, T &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    T incl = warp_inclusive_scan(v, lane);
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nwarps ? wsum[lane] : T(0);
        T wi = warp_inclusive_scan(w, lane);
        if (lane < nwarps) wsum[lane] = wi - w;
        if (lane == 31) wsum[32] = wi;
    }
    __syncthreads();
    total = wsum[32];
    return wsum[warp] + incl - v;
}

template <typename T>
__global__ __launch_bounds__(SCAN_THREADS) void scan_reduce_kernel(const T *__restrict__ in, uint64_t n,
                                                                    T *__restrict__ partial) {
    __shared__ T wsum[33];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
    T s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_IPT; k++) {
        uint64_t i = base + (uint64_t)k * SCAN_THREADS + threadIdx.x;
        if (i < n) s += in[i];
    }
    T total;
    block_exclusive_scan(s, wsum, total);
    if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

template <typename T>
__global__ __launch_bounds__(SCAN_THREADS) void scan_tiles_kernel(const T *in, T *out, uint64_t n,
                                                                   const T *__restrict__ tile_offsets,
                                                                   T *d_total) {
    __shared__ T tile[SCAN_TILE];
    __shared__ T wsum[33];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
#pragma unroll
    for (int k = 0; k < SCAN_IPT; k++) {
        int j = k * SCAN_THREADS + threadIdx.x;
        uint64_t i = base + j;
        tile[j] = i < n ? in[i] : T(0);
    }
    __syncthreads();
    T v[SCAN_IPT];
    T s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_IPT; k++) {
        v[k] = tile[threadIdx.x * SCAN_IPT + k];
        s += v[k];
    }
    T total;
    T run = block_exclusive_scan(s, wsum, total);
    const T off = tile_offsets ? tile_offsets[blockIdx.x] : T(0);
#pragma unroll
    for (int k = 0; k < SCAN_IPT; k++) {
        tile[threadIdx.x * SCAN_IPT + k] = off + run;
        run += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SCAN_IPT; k++) {
        int j = k * SCAN_THREADS + threadIdx.x;
        uint64_t i = base + j;
        if (i < n) out[i] = tile[j];
    }
    if (d_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *d_total = off + total;
}

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

// ------------------------------------------------------------ radix sort --
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_IPT = 16;
constexpr int RS_TILE = RS_THREADS * RS_IPT;  // 4096 items per tile
constexpr int RS_WARP_ITEMS = RS_TILE / RS_WARPS;

template <int KK>
__device__ __forceinline__ uint64_t sort_key(uint64_t it) {
    if (KK == SK_IDENT) return it;
    if (KK == SK_LOW32) return (uint32_t)it;
    return hash_pair((int32_t)(uint32_t)it, (int32_t)(uint32_t)(it >> 32));
}

template <int KK>
__global__ __launch_bounds__(RS_THREADS) void rs_upsweep_kernel(const uint64_t *__restrict__ in, uint32_t n,
                                                                 int shift, int bits,
                                                                 uint32_t *__restrict__ counts,
                                                                 uint32_t nblocks) {
    __shared__ uint32_t h[RS_WARPS][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t D = 1u << bits, dmask = D - 1;
    for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_THREADS) (&h[0][0])[i] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE + (uint64_t)warp * RS_WARP_ITEMS;
#pragma unroll 4
    for (int r = 0; r < RS_IPT; r++) {
        uint64_t idx = base + (uint64_t)r * 32 + lane;
        if (idx < n) {
            uint32_t d = (uint32_t)(sort_key<KK>(in[idx]) >> shift) & dmask;
            atomicAdd(&h[warp][d], 1u);
        }
    }
    __syncthreads();
    if ((uint32_t)threadIdx.x < D) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < RS_WARPS; w++) s += h[w][threadIdx.x];
        counts[(uint64_t)threadIdx.x * nblocks + blockIdx.x] = s;
    }
}

template <int KK>
__global__ __launch_bounds__(RS_THREADS) void rs_downsweep_kernel(const uint64_t *__restrict__ in,
                                                                   uint64_t *__restrict__ out, uint32_t n,
                                                                   int shift, int bits,
                                                                   const uint32_t *__restrict__ offs,
                                                                   uint32_t nblocks) {
    __shared__ uint64_t tile[RS_TILE];
    __shared__ uint32_t wcnt[RS_WARPS][256];
    __shared__ uint32_t bstart[256];
    __shared__ uint32_t goff[256];
    __shared__ uint32_t wsum[RS_WARPS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t D = 1u << bits, dmask = D - 1;
    for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_THREADS) (&wcnt[0][0])[i] = 0;
    __syncthreads();

    const uint64_t tile_base = (uint64_t)blockIdx.x * RS_TILE;
    const uint64_t base = tile_base + (uint64_t)warp * RS_WARP_ITEMS;
    const unsigned lt = lanemask_lt();
    uint64_t it[RS_IPT];
    uint32_t rk[RS_IPT];
#pragma unroll
    for (int r = 0; r < RS_IPT; r++) {
        const uint64_t idx = base + (uint64_t)r * 32 + lane;
        const bool valid = idx < n;
        it[r] = valid ? in[idx] : 0ull;
        const uint32_t d = valid ? ((uint32_t)(sort_key<KK>(it[r]) >> shift) & dmask) : 0u;
        unsigned peers = __ballot_sync(AMJ_FULL_MASK, valid);
        for (int b = 0; b < bits; b++) {
            const bool bit = (d >> b) & 1u;
            const unsigned bb = __ballot_sync(AMJ_FULL_MASK, bit);
            peers &= bit ? bb : ~bb;
        }
        const uint32_t rank = __popc(peers & lt);
        const uint32_t before = valid ? wcnt[warp][d] : 0u;
        __syncwarp();
        if (valid && rank == 0) wcnt[warp][d] = before + __popc(peers);
        __syncwarp();
        rk[r] = before + rank;
    }
    __syncthreads();
    uint32_t tot = 0;
    if ((uint32_t)threadIdx.x < D) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < RS_WARPS; w++) {
            uint32_t c = wcnt[w][threadIdx.x];
            wcnt[w][threadIdx.x] = run;
            run += c;
        }
        tot = run;
    }
    const uint32_t incl = warp_inclusive_scan(tot, lane);
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t woff = 0;
    for (int w = 0; w < warp; w++) woff += wsum[w];
    bstart[threadIdx.x] = woff + incl - tot;
    if ((uint32_t)threadIdx.x < D) goff[threadIdx.x] = offs[(uint64_t)threadIdx.x * nblocks + blockIdx.x];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_IPT; r++) {
        const uint64_t idx = base + (uint64_t)r * 32 + lane;
        if (idx < n) {
            const uint32_t d = (uint32_t)(sort_key<KK>(it[r]) >> shift) & dmask;
            tile[bstart[d] + wcnt[warp][d] + rk[r]] = it[r];
        }
    }
    __syncthreads();
    const uint64_t rem = n - tile_base;
    const uint32_t cnt = rem < (uint64_t)RS_TILE ? (uint32_t)rem : (uint32_t)RS_TILE;
    for (uint32_t i = threadIdx.x; i < cnt; i += RS_THREADS) {
        const uint64_t v = tile[i];
        const uint32_t d = (uint32_t)(sort_key<KK>(v) >> shift) & dmask;
        out[goff[d] + (i - bstart[d])] = v;
    }
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
