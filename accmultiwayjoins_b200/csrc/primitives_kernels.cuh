// Kernels of the device primitives (prefix sums, LSD radix sort), shared by
// the translation units that drive them with their own scratch memory.
#pragma once
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
__global__ __launch_bounds__(RS_THREADS, 3) void rs_downsweep_kernel(const uint64_t *__restrict__ in,
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
    // all of the thread's loads in flight before the ranking
#pragma unroll
    for (int r = 0; r < RS_IPT; r++) {
        const uint64_t idx = base + (uint64_t)r * 32 + lane;
        it[r] = idx < n ? in[idx] : 0ull;
    }
#pragma unroll
    for (int r = 0; r < RS_IPT; r++) {
        const uint64_t idx = base + (uint64_t)r * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = valid ? ((uint32_t)(sort_key<KK>(it[r]) >> shift) & dmask) : 0u;
        // lanes holding the same digit: one ballot per digit bit (cheaper
        // than a match on sm_100a: 2.07 against 2.51 ms for the C2 builds);
        // invalid lanes stay out of every valid lane's set
        unsigned peers = __ballot_sync(AMJ_FULL_MASK, valid);
#pragma unroll
        for (int b = 0; b < 8; b++) {
            if (b >= bits) break;
            const bool on = (d >> b) & 1u;
            const unsigned m = __ballot_sync(AMJ_FULL_MASK, on);
            peers &= on ? m : ~m;
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

}  // namespace amj
