// IndexedTrie construction and .tr (de)serialisation for 2-column relations.
//
// Reference: constructSortedTrie (LFTJ-GPU/multi_partitioning.cuh:129-293)
// sorts the tuples with CUB / Thrust, marks value changes (extractMasks,
// :104), and compacts the distinct values and their child offsets with
// segmented selects and scans.  Here: one min/max reduction sizes a compact
// sort key (c0 - min0) << bits1 | (c1 - min1) so the LSD radix sort runs only
// over the bits that vary (40 bits -> 5 passes for 2^20 vertices), then one
// kernel unpacks level 1 and flags group heads, a scan numbers the heads and
// a scatter writes level 0 and its offsets.  A dense row-pointer array over
// the level-0 value range is added when that range is small, so a probe can
// find a value's children with one load instead of a binary search.
#include "amj_ops.cuh"

#include <cstdio>
#include <cstring>
#include <vector>

namespace amj {

__global__ void minmax_pairs_kernel(const int32_t *__restrict__ c0, const int32_t *__restrict__ c1, uint64_t n,
                                    uint32_t *mm /* min0,max0,min1,max1 in sign-flipped order */) {
    uint32_t mn0 = 0xffffffffu, mx0 = 0, mn1 = 0xffffffffu, mx1 = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t a = (uint32_t)c0[i] ^ 0x80000000u, b = (uint32_t)c1[i] ^ 0x80000000u;
        mn0 = min(mn0, a); mx0 = max(mx0, a);
        mn1 = min(mn1, b); mx1 = max(mx1, b);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        mn0 = min(mn0, __shfl_xor_sync(AMJ_FULL_MASK, mn0, d));
        mx0 = max(mx0, __shfl_xor_sync(AMJ_FULL_MASK, mx0, d));
        mn1 = min(mn1, __shfl_xor_sync(AMJ_FULL_MASK, mn1, d));
        mx1 = max(mx1, __shfl_xor_sync(AMJ_FULL_MASK, mx1, d));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&mm[0], mn0); atomicMax(&mm[1], mx0);
        atomicMin(&mm[2], mn1); atomicMax(&mm[3], mx1);
    }
}

__global__ void pack_trie_keys_kernel(const int32_t *__restrict__ c0, const int32_t *__restrict__ c1, uint64_t n,
                                      uint32_t min0, uint32_t min1, int bits1, uint64_t *__restrict__ items) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t a = ((uint32_t)c0[i] ^ 0x80000000u) - min0;
        uint64_t b = ((uint32_t)c1[i] ^ 0x80000000u) - min1;
        items[i] = (a << bits1) | b;
    }
}

__device__ __forceinline__ int32_t unflip(uint64_t v, uint32_t mn) {
    return (int32_t)(((uint32_t)v + mn) ^ 0x80000000u);
}

__global__ void unpack_trie_kernel(const uint64_t *__restrict__ items, uint64_t n, uint32_t min0, uint32_t min1,
                                   int bits1, int32_t *__restrict__ data1, int32_t *__restrict__ src1,
                                   uint32_t *__restrict__ head) {
    const uint64_t m1 = bits1 >= 64 ? ~0ull : ((1ull << bits1) - 1);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = items[i];
        data1[i] = unflip(v & m1, min1);
        src1[i] = unflip(v >> bits1, min0);
        head[i] = (i == 0 || (items[i - 1] >> bits1) != (v >> bits1)) ? 1u : 0u;
    }
}

__global__ void scatter_level0_kernel(const uint64_t *__restrict__ items, const uint32_t *__restrict__ head,
                                      const uint32_t *__restrict__ pos, uint64_t n, uint32_t min0, int bits1,
                                      int32_t *__restrict__ data0, uint64_t *__restrict__ off0, uint64_t len0) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        // head[] was scanned in place into pos[]; recompute the head flag
        const bool h = (i == 0) || ((items[i - 1] >> bits1) != (items[i] >> bits1));
        if (h) {
            const uint32_t p = pos[i];
            data0[p] = unflip(items[i] >> bits1, min0);
            off0[p] = i;
        }
        if (i == 0) off0[len0] = n;
    }
    (void)head;
}

// adjacent equal items of a sorted array (duplicate rows), counted per block
__global__ void count_dups_kernel(const uint64_t *__restrict__ items, uint64_t n, unsigned long long *dups) {
    unsigned long long c = 0;
    for (uint64_t i = 1 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        c += items[i] == items[i - 1];
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(dups, c);
}

__global__ void first_of_run_kernel(const uint64_t *__restrict__ items, uint64_t n, uint32_t *__restrict__ flag) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || items[i] != items[i - 1]) ? 1u : 0u;
}

__global__ void compact_runs_kernel(const uint64_t *__restrict__ items, const uint32_t *__restrict__ pos, uint64_t n,
                                    uint64_t *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (i == 0 || items[i] != items[i - 1]) out[pos[i]] = items[i];
}

// child counts of every level-0 value, indexed densely by value - min
__global__ void dense_counts_kernel(const int32_t *__restrict__ data0, const uint64_t *__restrict__ off0,
                                    uint64_t len0, int32_t vmin, uint64_t *__restrict__ counts) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len0; i += (uint64_t)gridDim.x * blockDim.x)
        counts[(uint64_t)((int64_t)data0[i] - (int64_t)vmin)] = off0[i + 1] - off0[i];
}

static unsigned grid_for(amj_ctx *ctx, uint64_t n) {
    uint64_t g = (n + 255) / 256, cap = (uint64_t)ctx->num_sms * 16;
    return (unsigned)(g == 0 ? 1 : (g > cap ? cap : g));
}

static int bits_for(uint32_t range) {
    int b = 0;
    while (b < 32 && (range >> b) != 0) b++;
    return b;
}

int build_trie2(amj_ctx *ctx, const int32_t *d_c0, const int32_t *d_c1, uint64_t n, Trie2 *out, bool distinct,
                int32_t vmax) {
    if (n >= (1ull << 32) - 4096) return fail(AMJ_EUNSUPPORTED, "trie build: 2^32 or more rows");
    out->len1 = n;
    if (n == 0) {
        out->len0 = 0;
        AMJ_TRY(out->off0.alloc(ctx, 1));
        AMJ_CUDA_TRY(cudaMemsetAsync(out->off0.p, 0, sizeof(uint64_t), ctx->stream));
        AMJ_TRY(out->data0.alloc(ctx, 1));
        AMJ_TRY(out->data1.alloc(ctx, TRIE_LEVEL1_PAD));
        return AMJ_OK;
    }
    uint32_t h_mm[4];   // flipped min / max of both columns
    if (vmax >= 0) {
        // the caller knows every value lies in [0, vmax]
        h_mm[0] = h_mm[2] = 0x80000000u;
        h_mm[1] = h_mm[3] = (uint32_t)vmax ^ 0x80000000u;
    } else {
        DBuf<uint32_t> mm;
        AMJ_TRY(mm.alloc(ctx, 8));
        const uint32_t init[4] = {0xffffffffu, 0u, 0xffffffffu, 0u};
        AMJ_CUDA_TRY(cudaMemcpyAsync(mm.p, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
        note_launch(ctx);
        minmax_pairs_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(d_c0, d_c1, n, mm.p);
        AMJ_CUDA_TRY(cudaGetLastError());
        AMJ_CUDA_TRY(cudaMemcpyAsync(h_mm, mm.p, sizeof(h_mm), cudaMemcpyDeviceToHost, ctx->stream));
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    const uint32_t min0 = h_mm[0], min1 = h_mm[2];
    const int bits0 = bits_for(h_mm[1] - min0), bits1 = bits_for(h_mm[3] - min1);

    DBuf<uint64_t> a, b;
    AMJ_TRY(a.alloc(ctx, n));
    AMJ_TRY(b.alloc(ctx, n));
    note_launch(ctx);
    pack_trie_keys_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(d_c0, d_c1, n, min0, min1, bits1, a.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    uint64_t *sorted = nullptr;
    AMJ_TRY(radix_sort_u64(ctx, a.p, b.p, n, SK_IDENT, 0, bits0 + bits1, &sorted));
    // set semantics (distinct): repeated rows are adjacent after the sort;
    // they are counted beside the level-1 unpack and, when there are some,
    // dropped and the unpack redone
    DBuf<unsigned long long> dups;
    if (distinct && n > 1) {
        AMJ_TRY(dups.alloc(ctx, 1));
        AMJ_CUDA_TRY(cudaMemsetAsync(dups.p, 0, sizeof(unsigned long long), ctx->stream));
        note_launch(ctx);
        count_dups_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sorted, n, dups.p);
        AMJ_CUDA_TRY(cudaGetLastError());
    }
    AMJ_TRY(out->data1.alloc(ctx, n + TRIE_LEVEL1_PAD));
    AMJ_TRY(out->src1.alloc(ctx, n));
    DBuf<uint32_t> head;
    AMJ_TRY(head.alloc(ctx, n + 1));
    uint32_t len0 = 0;
    unsigned long long h_dups = 0;
    for (int round = 0; round < 2; round++) {
        note_launch(ctx);
        unpack_trie_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sorted, n, min0, min1, bits1, out->data1.p,
                                                                       out->src1.p, head.p);
        AMJ_CUDA_TRY(cudaGetLastError());
        AMJ_TRY(scan_exclusive_u32(ctx, head.p, head.p, n, head.p + n));
        AMJ_CUDA_TRY(cudaMemcpyAsync(&len0, head.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
        if (round == 0 && dups.p)
            AMJ_CUDA_TRY(cudaMemcpyAsync(&h_dups, dups.p, sizeof(h_dups), cudaMemcpyDeviceToHost, ctx->stream));
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (round > 0 || h_dups == 0) break;
        DBuf<uint32_t> pos;
        AMJ_TRY(pos.alloc(ctx, n));
        note_launch(ctx);
        first_of_run_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sorted, n, pos.p);
        AMJ_CUDA_TRY(cudaGetLastError());
        AMJ_TRY(scan_exclusive_u32(ctx, pos.p, pos.p, n, nullptr));
        uint64_t *other = sorted == a.p ? b.p : a.p;
        note_launch(ctx);
        compact_runs_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sorted, pos.p, n, other);
        AMJ_CUDA_TRY(cudaGetLastError());
        sorted = other;
        n -= h_dups;
        out->len1 = n;
    }
    out->len0 = len0;
    AMJ_TRY(out->data0.alloc(ctx, len0));
    AMJ_TRY(out->off0.alloc(ctx, (uint64_t)len0 + 1));
    note_launch(ctx);
    scatter_level0_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sorted, head.p, head.p, n, min0, bits1,
                                                                      out->data0.p, out->off0.p, len0);
    AMJ_CUDA_TRY(cudaGetLastError());
    // dense row pointers when the level-0 value range is small against the trie
    const uint64_t range = (uint64_t)(h_mm[1] - min0) + 1;
    if (range <= 4 * (uint64_t)len0 + 4096 && range < (1ull << 31)) {
        out->rp_min = (int32_t)(min0 ^ 0x80000000u);
        out->rp_count = range;
        AMJ_TRY(out->rowptr.alloc(ctx, range + 1));
        AMJ_CUDA_TRY(cudaMemsetAsync(out->rowptr.p, 0, (range + 1) * sizeof(uint64_t), ctx->stream));
        note_launch(ctx);
        dense_counts_kernel<<<grid_for(ctx, len0), 256, 0, ctx->stream>>>(out->data0.p, out->off0.p, len0,
                                                                          out->rp_min, out->rowptr.p);
        AMJ_CUDA_TRY(cudaGetLastError());
        AMJ_TRY(scan_exclusive_u64(ctx, out->rowptr.p, out->rowptr.p, range + 1, nullptr));
    }
    return AMJ_OK;
}

// ---- 2-level tries of a degree-ranked copy: rows by counting ----
// Every value lies in [0, nv) and every row's first value is below its
// second, so the rows can be bucketed by their first value directly: a count
// per value, a scan into row starts, and one scatter of the second values
// into their rows, then each row sorted on its own.  After the degree
// ranking a row holds the higher-ranked neighbours of one vertex, at most
// sqrt(2 n) of them, and most rows hold a few: a warp sorts a row of up to
// 32 values in registers (a bitonic network over shuffles) and up to
// RK_WARP_MAX in its shared-memory slice; a block sorts the longer rows, up to
// RK_BLOCK_MAX.  A graph with a longer row takes the radix-sort build.
// Repeated rows (adjacent after the sort) are dropped by a compaction pass
// when there are any.
constexpr uint32_t RK_WARP_MAX = 1024;
constexpr uint32_t RK_BLOCK_MAX = 8192;
constexpr int RK_SORT_WARPS = 8;

__global__ void rk_count_kernel(const int32_t *__restrict__ c0, uint64_t n, uint32_t *__restrict__ cnt) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[c0[i]], 1u);
}

__global__ void rk_max_kernel(const uint32_t *__restrict__ cnt, uint64_t nv, unsigned int *__restrict__ mx) {
    uint32_t m = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < nv; v += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, cnt[v]);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) m = max(m, __shfl_xor_sync(AMJ_FULL_MASK, m, d));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(mx, m);
}

// fill[] starts at zero: the row of value c0[i] gets c1[i] at its next free slot
__global__ void rk_scatter_kernel(const int32_t *__restrict__ c0, const int32_t *__restrict__ c1, uint64_t n,
                                  const uint32_t *__restrict__ start, uint32_t *__restrict__ fill,
                                  int32_t *__restrict__ data1) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const int32_t v = c0[i];
        data1[start[v] + atomicAdd(&fill[v], 1u)] = c1[i];
    }
}

// ascending bitonic sort of the pow2-sized x[0, m) by the threads t of a
// group of nt, with sync() between stages
template <class Sync>
__device__ __forceinline__ void rk_bitonic(int32_t *x, uint32_t m, uint32_t t, uint32_t nt, Sync &&sync) {
    for (uint32_t k = 2; k <= m; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = t; i < m; i += nt) {
                const uint32_t p = i ^ j;
                if (p > i) {
                    const int32_t a = x[i], b = x[p];
                    if ((a > b) == ((i & k) == 0)) {
                        x[i] = b;
                        x[p] = a;
                    }
                }
            }
            sync();
        }
}

// distinct values of the sorted row x[0, len) (shared memory), counted by a group
__device__ __forceinline__ uint32_t rk_distinct(const int32_t *x, uint32_t len, uint32_t t, uint32_t nt) {
    uint32_t u = 0;
    for (uint32_t i = t; i < len; i += nt) u += (i == 0 || x[i] != x[i - 1]) ? 1u : 0u;
    return u;
}

// A row of up to 32 E values sorted by one warp in registers: value i of the
// sorted row ends in register i % E of lane i / E.  The values may start in
// any lanes and registers.  A bitonic network: a stage whose partner distance
// j is E or more exchanges registers between lanes (shuffles), a shorter one
// within a lane.
template <int E>
__device__ __forceinline__ void rk_warp_bitonic(int32_t (&x)[E], uint32_t lane) {
#pragma unroll
    for (uint32_t k = 2; k <= 32u * E; k <<= 1)
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            if (j >= (uint32_t)E) {
                const uint32_t lj = j / E;
                const bool lower = (lane & lj) == 0;
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const bool up = ((lane * E + e) & k) == 0;
                    const int32_t y = __shfl_xor_sync(AMJ_FULL_MASK, x[e], lj);
                    x[e] = (lower == up) ? min(x[e], y) : max(x[e], y);
                }
            } else {
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const int p = e ^ (int)j;
                    if (p > e) {
                        const bool up = ((lane * E + e) & k) == 0;
                        const int32_t a = x[e], b = x[p];
                        x[e] = up ? min(a, b) : max(a, b);
                        x[p] = up ? max(a, b) : min(a, b);
                    }
                }
            }
        }
}

// row v = data1[s, s + len), 32 (E / 2) < len <= 32 E: sorted in place, its
// level-0 value into src1, its number of distinct values into uniq[v]
template <int E>
__device__ __forceinline__ void rk_warp_row(int32_t *__restrict__ data1, int32_t *__restrict__ src1,
                                            uint32_t *__restrict__ uniq, uint32_t s, uint32_t len, uint64_t v,
                                            uint32_t lane) {
    int32_t x[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
        const uint32_t i = e * 32u + lane;   // coalesced loads; the network fixes the order
        x[e] = i < len ? data1[s + i] : INT32_MAX;
    }
    rk_warp_bitonic<E>(x, lane);
    const int32_t prev = __shfl_up_sync(AMJ_FULL_MASK, x[E - 1], 1);
    uint32_t u = 0;
#pragma unroll
    for (int e = 0; e < E; e++) {
        const uint32_t i = lane * E + e;
        if (i < len) {
            const int32_t before = e ? x[e - 1] : prev;
            u += (i == 0 || x[e] != before) ? 1u : 0u;
            data1[s + i] = x[e];
            src1[s + i] = (int32_t)v;
        }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) u += __shfl_xor_sync(AMJ_FULL_MASK, u, d);
    if (lane == 0) uniq[v] = u;
}

// One warp a row, the row's values in registers (rows of up to RK_WARP_MAX);
// longer rows are listed for the block kernel.
__global__ __launch_bounds__(RK_SORT_WARPS * 32, 4) void rk_sort_rows_kernel(const uint32_t *__restrict__ start,
                                                                           uint64_t nv, int32_t *__restrict__ data1,
                                                                           int32_t *__restrict__ src1,
                                                                           uint32_t *__restrict__ uniq,
                                                                           uint32_t *__restrict__ longs,
                                                                           unsigned int *__restrict__ nlong) {
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t warps = (uint64_t)gridDim.x * RK_SORT_WARPS;
    for (uint64_t v = blockIdx.x * (uint64_t)RK_SORT_WARPS + w; v < nv; v += warps) {
        const uint32_t s = start[v], len = start[v + 1] - s;
        if (len <= 1) {
            if (len == 1 && lane == 0) src1[s] = (int32_t)v;
            if (lane == 0) uniq[v] = len;
        } else if (len <= 32) {
            rk_warp_row<1>(data1, src1, uniq, s, len, v, lane);
        } else if (len <= 64) {
            rk_warp_row<2>(data1, src1, uniq, s, len, v, lane);
        } else if (len <= 128) {
            rk_warp_row<4>(data1, src1, uniq, s, len, v, lane);
        } else if (len <= 256) {
            rk_warp_row<8>(data1, src1, uniq, s, len, v, lane);
        } else if (len <= 512) {
            rk_warp_row<16>(data1, src1, uniq, s, len, v, lane);
        } else if (len <= RK_WARP_MAX) {
            rk_warp_row<32>(data1, src1, uniq, s, len, v, lane);
        } else if (lane == 0) {
            longs[atomicAdd(nlong, 1u)] = (uint32_t)v;
            uniq[v] = 0;
        }
    }
}

// One block a listed row (RK_WARP_MAX < length <= RK_BLOCK_MAX); the blocks
// take the list's rows in turn
__global__ __launch_bounds__(512) void rk_sort_long_kernel(const uint32_t *__restrict__ start,
                                                           int32_t *__restrict__ data1, int32_t *__restrict__ src1,
                                                           uint32_t *__restrict__ uniq,
                                                           const uint32_t *__restrict__ longs,
                                                           const unsigned int *__restrict__ nlong) {
    __shared__ int32_t x[RK_BLOCK_MAX];
    __shared__ uint32_t usum;
    const uint32_t t = threadIdx.x, nt = blockDim.x;
    for (uint32_t r = blockIdx.x; r < *nlong; r += gridDim.x) {
        const uint32_t v = longs[r], s = start[v], len = start[v + 1] - s;
        uint32_t m = 64;
        while (m < len) m <<= 1;
        if (t == 0) usum = 0;
        for (uint32_t i = t; i < m; i += nt) x[i] = i < len ? data1[s + i] : INT32_MAX;
        __syncthreads();
        rk_bitonic(x, m, t, nt, [] { __syncthreads(); });
        const uint32_t u = rk_distinct(x, len, t, nt);
        if (u) atomicAdd(&usum, u);
        for (uint32_t i = t; i < len; i += nt) {
            data1[s + i] = x[i];
            src1[s + i] = (int32_t)v;
        }
        __syncthreads();
        if (t == 0) uniq[v] = usum;
        __syncthreads();
    }
}

// repeated rows present: row v's distinct values move to ustart[v] (a warp a row)
__global__ void rk_compact_kernel(const uint32_t *__restrict__ start, const uint32_t *__restrict__ ustart,
                                  uint64_t nv, const int32_t *__restrict__ data1, int32_t *__restrict__ out1,
                                  int32_t *__restrict__ outsrc) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < nv; v += warps) {
        const uint32_t s = start[v], len = start[v + 1] - s;
        uint32_t at = ustart[v];
        for (uint32_t i0 = 0; i0 < len; i0 += 32) {
            const uint32_t i = i0 + lane;
            const bool keep = i < len && (i == 0 || data1[s + i] != data1[s + i - 1]);
            const unsigned b = __ballot_sync(AMJ_FULL_MASK, keep);
            if (keep) {
                const uint32_t o = at + __popc(b & ((1u << lane) - 1u));
                out1[o] = data1[s + i];
                outsrc[o] = (int32_t)v;
            }
            at += __popc(b);
        }
    }
}

// level 0 (the values with children) and the dense row pointers
__global__ void rk_level0_kernel(const uint32_t *__restrict__ ustart, const uint32_t *__restrict__ pos, uint64_t nv,
                                 int32_t *__restrict__ data0, uint64_t *__restrict__ off0,
                                 uint64_t *__restrict__ rowptr, uint64_t len0) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v <= nv; v += (uint64_t)gridDim.x * blockDim.x) {
        rowptr[v] = ustart[v];
        if (v == nv) {
            off0[len0] = ustart[nv];
        } else if (ustart[v + 1] > ustart[v]) {
            data0[pos[v]] = (int32_t)v;
            off0[pos[v]] = ustart[v];
        }
    }
}

// 1 for the values with a row (every row keeps a value after deduplication)
__global__ void rk_nonempty_kernel(const uint32_t *__restrict__ start, uint64_t nv, uint32_t *__restrict__ flag) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < nv; v += (uint64_t)gridDim.x * blockDim.x)
        flag[v] = start[v + 1] > start[v] ? 1u : 0u;
}

int build_trie2_ranked(amj_ctx *ctx, const int32_t *d_c0, const int32_t *d_c1, uint64_t n, uint64_t nv, Trie2 *out) {
    if (n == 0 || nv == 0 || nv >= (1ull << 31) || n >= (1ull << 32) - 4096)
        return build_trie2(ctx, d_c0, d_c1, n, out, true, nv ? (int32_t)(nv - 1) : -1);
    // per-value row lengths, the longest, the row starts, and the values with
    // children (level 0) numbered by a scan of their flags
    DBuf<uint32_t> start, fill, flag;
    DBuf<unsigned int> ctr;   // [0] longest row, [1] rows listed for the block kernel
    AMJ_TRY(start.alloc(ctx, nv + 1));
    AMJ_TRY(fill.alloc(ctx, nv));
    AMJ_TRY(flag.alloc(ctx, nv + 1));
    AMJ_TRY(ctr.alloc(ctx, 2));
    AMJ_CUDA_TRY(cudaMemsetAsync(start.p, 0, (nv + 1) * sizeof(uint32_t), ctx->stream));
    AMJ_CUDA_TRY(cudaMemsetAsync(ctr.p, 0, 2 * sizeof(unsigned int), ctx->stream));
    note_launch(ctx);
    rk_count_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(d_c0, n, start.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    note_launch(ctx);
    rk_max_kernel<<<grid_for(ctx, nv), 256, 0, ctx->stream>>>(start.p, nv, ctr.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_TRY(scan_exclusive_u32(ctx, start.p, start.p, nv + 1, nullptr));
    note_launch(ctx);
    rk_nonempty_kernel<<<grid_for(ctx, nv), 256, 0, ctx->stream>>>(start.p, nv, flag.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_TRY(scan_exclusive_u32(ctx, flag.p, flag.p, nv, flag.p + nv));
    uint32_t h[2] = {0, 0};   // longest row, values with children
    AMJ_CUDA_TRY(cudaMemcpyAsync(&h[0], ctr.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaMemcpyAsync(&h[1], flag.p + nv, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    const uint32_t longest = h[0], len0 = h[1];
    if (longest > RK_BLOCK_MAX) return build_trie2(ctx, d_c0, d_c1, n, out, true, (int32_t)(nv - 1));
    // the rows, each sorted, with their distinct counts
    AMJ_TRY(out->data1.alloc(ctx, n + TRIE_LEVEL1_PAD));
    AMJ_TRY(out->src1.alloc(ctx, n));
    DBuf<uint32_t> uniq, longs;
    AMJ_TRY(uniq.alloc(ctx, nv + 1));
    AMJ_TRY(longs.alloc(ctx, std::max<uint64_t>(1, n / (RK_WARP_MAX + 1) + 1)));
    AMJ_CUDA_TRY(cudaMemsetAsync(fill.p, 0, nv * sizeof(uint32_t), ctx->stream));
    note_launch(ctx);
    rk_scatter_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(d_c0, d_c1, n, start.p, fill.p, out->data1.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    const unsigned gs = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((nv + RK_SORT_WARPS - 1) / RK_SORT_WARPS,
                                                                           (uint64_t)ctx->num_sms * 8));
    note_launch(ctx);
    rk_sort_rows_kernel<<<gs, RK_SORT_WARPS * 32, 0, ctx->stream>>>(start.p, nv, out->data1.p, out->src1.p, uniq.p,
                                                                    longs.p, ctr.p + 1);
    AMJ_CUDA_TRY(cudaGetLastError());
    if (longest > RK_WARP_MAX) {
        note_launch(ctx);
        rk_sort_long_kernel<<<ctx->num_sms, 512, 0, ctx->stream>>>(start.p, out->data1.p, out->src1.p, uniq.p,
                                                                   longs.p, ctr.p + 1);
        AMJ_CUDA_TRY(cudaGetLastError());
    }
    // distinct rows: scan the distinct counts; a compaction when some differ
    uint32_t h_total = 0;
    AMJ_TRY(scan_exclusive_u32(ctx, uniq.p, uniq.p, nv + 1, nullptr));
    AMJ_CUDA_TRY(cudaMemcpyAsync(&h_total, uniq.p + nv, sizeof(h_total), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (h_total != n) {
        DBuf<int32_t> d1, s1;
        AMJ_TRY(d1.alloc(ctx, (uint64_t)h_total + TRIE_LEVEL1_PAD));
        AMJ_TRY(s1.alloc(ctx, h_total ? h_total : 1));
        note_launch(ctx);
        rk_compact_kernel<<<grid_for(ctx, nv * 32), 256, 0, ctx->stream>>>(start.p, uniq.p, nv, out->data1.p, d1.p,
                                                                            s1.p);
        AMJ_CUDA_TRY(cudaGetLastError());
        out->data1 = std::move(d1);
        out->src1 = std::move(s1);
    }
    out->len1 = h_total;
    // level 0 and the dense row pointers (a row with values keeps at least one)
    out->len0 = len0;
    AMJ_TRY(out->data0.alloc(ctx, len0 ? len0 : 1));
    AMJ_TRY(out->off0.alloc(ctx, (uint64_t)len0 + 1));
    AMJ_TRY(out->rowptr.alloc(ctx, nv + 1));
    out->rp_min = 0;
    out->rp_count = nv;
    note_launch(ctx);
    rk_level0_kernel<<<grid_for(ctx, nv + 1), 256, 0, ctx->stream>>>(uniq.p, flag.p, nv, out->data0.p, out->off0.p,
                                                                     out->rowptr.p, len0);
    AMJ_CUDA_TRY(cudaGetLastError());
    return AMJ_OK;
}

// ---- N-level tries ----
// Rows are ordered by a stable LSD radix sort of the row permutation, one
// column at a time from the last: items (column value - min) << 32 | row,
// sorted on the value bits only.  Then per level a head flag marks the rows
// whose (l+1)-prefix differs from the previous row's, a scan numbers the
// heads, and a scatter writes the level's values and child offsets.

__global__ void minmax_col_kernel(const int32_t *__restrict__ c, uint64_t n, uint32_t *mm) {
    uint32_t mn = 0xffffffffu, mx = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = (uint32_t)c[i] ^ 0x80000000u;
        mn = min(mn, a);
        mx = max(mx, a);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        mn = min(mn, __shfl_xor_sync(AMJ_FULL_MASK, mn, d));
        mx = max(mx, __shfl_xor_sync(AMJ_FULL_MASK, mx, d));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&mm[0], mn);
        atomicMax(&mm[1], mx);
    }
}

__global__ void pack_col_kernel(const int32_t *__restrict__ c, const uint32_t *__restrict__ perm, uint64_t n,
                                uint32_t mn, uint64_t *__restrict__ items) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = perm ? perm[i] : (uint32_t)i;
        items[i] = ((uint64_t)(((uint32_t)c[r] ^ 0x80000000u) - mn) << 32) | r;
    }
}

__global__ void perm_from_items_kernel(const uint64_t *__restrict__ items, uint64_t n, uint32_t *__restrict__ perm) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        perm[i] = (uint32_t)items[i];
}

__global__ void gather_perm_kernel(const int32_t *__restrict__ c, const uint32_t *__restrict__ perm, uint64_t n,
                                   int32_t *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = c[perm ? perm[i] : i];
}

// head[i] = 1 when row i's (l+1)-prefix differs from row i-1's
__global__ void prefix_heads_kernel(int32_t *const *__restrict__ S, int l, uint64_t n, uint32_t *__restrict__ head) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        bool h = i == 0;
        for (int c = 0; c <= l && !h; c++) h = S[c][i] != S[c][i - 1];
        head[i] = h ? 1u : 0u;
    }
}

// level l: values and child offsets at the heads' ranks
__global__ void scatter_level_kernel(const int32_t *__restrict__ Sl, const uint32_t *__restrict__ head,
                                     const uint32_t *__restrict__ rank, const uint32_t *__restrict__ next_rank,
                                     uint64_t n, int32_t *__restrict__ data, uint64_t *__restrict__ off) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        const uint32_t r = rank[i];
        data[r] = Sl[i];
        off[r] = next_rank ? next_rank[i] : i;
    }
}

int build_trieN(amj_ctx *ctx, const int32_t *const *d_cols, int ncols, uint64_t n, TrieN *out) {
    if (ncols < 1 || ncols > TRIE_MAX_LEVELS) return fail(AMJ_EINVAL, "trie_build_n: 1..8 columns");
    if (n >= (1ull << 32)) return fail(AMJ_EUNSUPPORTED, "trie_build_n: 2^32 or more rows");
    out->levels = ncols;
    // sorted columns
    std::vector<DBuf<int32_t>> S(ncols);
    DBuf<uint32_t> perm;
    if (n > 1) {
        DBuf<uint64_t> a, b;
        DBuf<uint32_t> mm;
        AMJ_TRY(a.alloc(ctx, n));
        AMJ_TRY(b.alloc(ctx, n));
        AMJ_TRY(perm.alloc(ctx, n));
        AMJ_TRY(mm.alloc(ctx, 2 * ncols));
        std::vector<uint32_t> init(2 * ncols);
        for (int c = 0; c < ncols; c++) {
            init[2 * c] = 0xffffffffu;
            init[2 * c + 1] = 0;
        }
        AMJ_CUDA_TRY(cudaMemcpyAsync(mm.p, init.data(), 8 * ncols, cudaMemcpyHostToDevice, ctx->stream));
        for (int c = 0; c < ncols; c++) {
            note_launch(ctx);
            minmax_col_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(d_cols[c], n, mm.p + 2 * c);
        }
        AMJ_CUDA_TRY(cudaGetLastError());
        std::vector<uint32_t> h(2 * ncols);
        AMJ_CUDA_TRY(cudaMemcpyAsync(h.data(), mm.p, 8 * ncols, cudaMemcpyDeviceToHost, ctx->stream));
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        bool have_perm = false;
        for (int c = ncols - 1; c >= 0; c--) {
            const uint32_t range = h[2 * c + 1] - h[2 * c];
            int bits = 0;
            while (bits < 32 && (uint64_t)range >> bits) bits++;
            if (bits == 0) continue;   // constant column: the order stays
            note_launch(ctx);
            pack_col_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(d_cols[c], have_perm ? perm.p : nullptr, n,
                                                                      h[2 * c], a.p);
            AMJ_CUDA_TRY(cudaGetLastError());
            uint64_t *sorted = nullptr;
            AMJ_TRY(radix_sort_u64(ctx, a.p, b.p, n, SK_IDENT, 32, 32 + bits, &sorted));
            note_launch(ctx);
            perm_from_items_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sorted, n, perm.p);
            AMJ_CUDA_TRY(cudaGetLastError());
            have_perm = true;
        }
        if (!have_perm) perm.release();
    }
    for (int c = 0; c < ncols; c++) {
        AMJ_TRY(S[c].alloc(ctx, n ? n : 1));
        if (n) {
            note_launch(ctx);
            gather_perm_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(d_cols[c], perm.p, n, S[c].p);
        }
    }
    AMJ_CUDA_TRY(cudaGetLastError());
    // heads and ranks of every level but the last
    const int L = ncols - 1;
    std::vector<DBuf<uint32_t>> head(L), rank(L);
    std::vector<uint32_t> cnt(L, 0);
    DBuf<int32_t *> sp;
    AMJ_TRY(sp.alloc(ctx, ncols));
    std::vector<int32_t *> hp(ncols);
    for (int c = 0; c < ncols; c++) hp[c] = S[c].p;
    AMJ_CUDA_TRY(cudaMemcpyAsync(sp.p, hp.data(), ncols * sizeof(int32_t *), cudaMemcpyHostToDevice, ctx->stream));
    DBuf<uint32_t> totals;
    AMJ_TRY(totals.alloc(ctx, L ? L : 1));
    for (int l = 0; l < L; l++) {
        AMJ_TRY(head[l].alloc(ctx, n ? n : 1));
        AMJ_TRY(rank[l].alloc(ctx, n ? n : 1));
        if (n) {
            note_launch(ctx);
            prefix_heads_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(sp.p, l, n, head[l].p);
            AMJ_CUDA_TRY(cudaGetLastError());
            AMJ_TRY(scan_exclusive_u32(ctx, head[l].p, rank[l].p, n, totals.p + l));
        } else {
            AMJ_CUDA_TRY(cudaMemsetAsync(totals.p + l, 0, 4, ctx->stream));
        }
    }
    if (L) {
        AMJ_CUDA_TRY(cudaMemcpyAsync(cnt.data(), totals.p, 4 * L, cudaMemcpyDeviceToHost, ctx->stream));
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    for (int l = 0; l < L; l++) {
        out->len[l] = cnt[l];
        AMJ_TRY(out->data[l].alloc(ctx, cnt[l] ? cnt[l] : 1));
        AMJ_TRY(out->off[l].alloc(ctx, (uint64_t)cnt[l] + 1));
        if (n) {
            note_launch(ctx);
            scatter_level_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(
                S[l].p, head[l].p, rank[l].p, l + 1 < L ? rank[l + 1].p : nullptr, n, out->data[l].p, out->off[l].p);
            AMJ_CUDA_TRY(cudaGetLastError());
        }
        const uint64_t end = l + 1 < L ? (uint64_t)cnt[l + 1] : n;
        AMJ_CUDA_TRY(cudaMemcpyAsync(out->off[l].p + cnt[l], &end, 8, cudaMemcpyHostToDevice, ctx->stream));
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    out->len[L] = n;
    out->data[L] = std::move(S[L]);
    return AMJ_OK;
}

}  // namespace amj

using namespace amj;

extern "C" int amj_trie_download_level(const amj_trie *t, int level, int32_t *data, uint64_t *offsets);
extern "C" int amj_trie_save_n(const amj_trie *t, const char *path, const uint32_t *attrs);

extern "C" int amj_trie_build(amj_ctx *ctx, const int32_t *d_c0, const int32_t *d_c1, uint64_t n, amj_trie **out) {
    if (!ctx || !out || (n && (!d_c0 || !d_c1))) return fail(AMJ_EINVAL, "trie_build: null argument");
    *out = nullptr;
    auto *t = new amj_trie();
    t->ctx = ctx;
    int rc = build_trie2(ctx, d_c0, d_c1, n, &t->t);
    if (rc == AMJ_OK) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "trie_build");
    }
    if (rc != AMJ_OK) {
        delete t;
        return rc;
    }
    *out = t;
    return AMJ_OK;
}

extern "C" int amj_trie_view(const amj_trie *t, uint64_t *len0, uint64_t *len1, const int32_t **d_data0,
                             const uint64_t **d_offsets0, const int32_t **d_data1) {
    if (!t) return fail(AMJ_EINVAL, "trie_view: null trie");
    if (t->levels() != 2) return fail(AMJ_EINVAL, "trie_view: not a 2-level trie");
    if (len0) *len0 = t->len(0);
    if (len1) *len1 = t->len(1);
    if (d_data0) *d_data0 = t->data(0);
    if (d_offsets0) *d_offsets0 = t->off(0);
    if (d_data1) *d_data1 = t->data(1);
    return AMJ_OK;
}

extern "C" int amj_trie_download(const amj_trie *t, int32_t *data0, uint64_t *offsets0, int32_t *data1) {
    if (!t || !data0 || !offsets0 || !data1) return fail(AMJ_EINVAL, "trie_download: null argument");
    if (t->levels() != 2) return fail(AMJ_EINVAL, "trie_download: not a 2-level trie");
    AMJ_TRY(amj_trie_download_level(t, 0, data0, offsets0));
    return amj_trie_download_level(t, 1, data1, nullptr);
}

extern "C" void amj_trie_release(amj_trie *t) {
    if (!t) return;
    if (t->ctx) (void)cudaSetDevice(t->ctx->device);
    delete t;
}

// .tr layout (LFTJ-GPU/IndexedTrie.cuh:122-156): uint32 num_attrs, uint64
// data_len[num_attrs], uint32 attr_list[num_attrs], the int32 data of each
// level, then the uint64 offsets of every level but the last
// (data_len[l]+1 entries each).
extern "C" int amj_trie_save(const amj_trie *t, const char *path, uint32_t a0, uint32_t a1) {
    if (!t || !path) return fail(AMJ_EINVAL, "trie_save: null argument");
    if (t->levels() != 2) return fail(AMJ_EINVAL, "trie_save: not a 2-level trie");
    const uint32_t attrs[2] = {a0, a1};
    return amj_trie_save_n(t, path, attrs);
}

extern "C" int amj_trie_load(amj_ctx *ctx, const char *path, amj_trie **out, uint32_t *a0, uint32_t *a1) {
    if (!ctx || !path || !out) return fail(AMJ_EINVAL, "trie_load: null argument");
    *out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(AMJ_EIO, std::string("trie_load: cannot open ") + path);
    uint32_t na = 0;
    uint64_t lens[2] = {0, 0};
    uint32_t attrs[2] = {0, 0};
    if (std::fread(&na, 4, 1, f) != 1 || na != 2 || std::fread(lens, 8, 2, f) != 2 || std::fread(attrs, 4, 2, f) != 2) {
        std::fclose(f);
        return fail(AMJ_EIO, "trie_load: bad header (only 2-level tries are supported)");
    }
    const uint64_t l0 = lens[0], l1 = lens[1];
    std::vector<int32_t> d0(l0), d1(l1);
    std::vector<uint64_t> o0(l0 + 1);
    bool ok = (l0 == 0 || std::fread(d0.data(), 4, l0, f) == l0) && (l1 == 0 || std::fread(d1.data(), 4, l1, f) == l1) &&
              std::fread(o0.data(), 8, l0 + 1, f) == l0 + 1;
    std::fclose(f);
    if (!ok || o0[l0] != l1) return fail(AMJ_EIO, "trie_load: truncated or inconsistent file");
    auto *t = new amj_trie();
    t->ctx = ctx;
    t->t.len0 = l0;
    t->t.len1 = l1;
    int rc = t->t.data0.alloc(ctx, l0 ? l0 : 1);
    if (rc == AMJ_OK) rc = t->t.data1.alloc(ctx, l1 ? l1 : 1);
    if (rc == AMJ_OK) rc = t->t.off0.alloc(ctx, l0 + 1);
    if (rc == AMJ_OK && l0 && cudaMemcpyAsync(t->t.data0.p, d0.data(), l0 * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) rc = AMJ_ECUDA;
    if (rc == AMJ_OK && l1 && cudaMemcpyAsync(t->t.data1.p, d1.data(), l1 * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) rc = AMJ_ECUDA;
    if (rc == AMJ_OK && cudaMemcpyAsync(t->t.off0.p, o0.data(), (l0 + 1) * 8, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) rc = AMJ_ECUDA;
    if (rc == AMJ_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = AMJ_ECUDA;
    if (rc != AMJ_OK) {
        (void)cudaGetLastError();
        delete t;
        return rc == AMJ_ECUDA ? fail(rc, "trie_load: device copy failed") : rc;
    }
    if (a0) *a0 = attrs[0];
    if (a1) *a1 = attrs[1];
    *out = t;
    return AMJ_OK;
}

extern "C" int amj_trie_build_n(amj_ctx *ctx, const int32_t *const *d_cols, int ncols, uint64_t n, amj_trie **out) {
    if (!ctx || !out || !d_cols) return fail(AMJ_EINVAL, "trie_build_n: null argument");
    if (ncols < 1 || ncols > TRIE_MAX_LEVELS) return fail(AMJ_EINVAL, "trie_build_n: 1..8 columns");
    for (int c = 0; c < ncols && n; c++)
        if (!d_cols[c]) return fail(AMJ_EINVAL, "trie_build_n: null column");
    *out = nullptr;
    auto *t = new amj_trie();
    t->ctx = ctx;
    int rc = build_trieN(ctx, d_cols, ncols, n, &t->tn);
    if (rc == AMJ_OK) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "trie_build_n");
    }
    if (rc != AMJ_OK) {
        delete t;
        return rc;
    }
    *out = t;
    return AMJ_OK;
}

extern "C" int amj_trie_info(const amj_trie *t, int *levels, uint64_t *lens) {
    if (!t) return fail(AMJ_EINVAL, "trie_info: null trie");
    if (levels) *levels = t->levels();
    if (lens)
        for (int l = 0; l < t->levels(); l++) lens[l] = t->len(l);
    return AMJ_OK;
}

extern "C" int amj_trie_download_level(const amj_trie *t, int level, int32_t *data, uint64_t *offsets) {
    if (!t || !data) return fail(AMJ_EINVAL, "trie_download_level: null argument");
    if (level < 0 || level >= t->levels()) return fail(AMJ_EINVAL, "trie_download_level: no such level");
    amj_ctx *ctx = t->ctx;
    const uint64_t n = t->len(level);
    if (n) AMJ_CUDA_TRY(cudaMemcpyAsync(data, t->data(level), n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (offsets && level + 1 < t->levels())
        AMJ_CUDA_TRY(cudaMemcpyAsync(offsets, t->off(level), (n + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return AMJ_OK;
}

// .tr with any number of levels (same layout as amj_trie_save)
extern "C" int amj_trie_save_n(const amj_trie *t, const char *path, const uint32_t *attrs) {
    if (!t || !path || !attrs) return fail(AMJ_EINVAL, "trie_save_n: null argument");
    const int L = t->levels();
    std::vector<std::vector<int32_t>> d(L);
    std::vector<std::vector<uint64_t>> o(L > 1 ? L - 1 : 0);
    for (int l = 0; l < L; l++) {
        d[l].resize(t->len(l));
        if (l + 1 < L) o[l].resize(t->len(l) + 1);
        AMJ_TRY(amj_trie_download_level(t, l, d[l].data(), l + 1 < L ? o[l].data() : nullptr));
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(AMJ_EIO, std::string("trie_save_n: cannot open ") + path);
    const uint32_t na = (uint32_t)L;
    bool ok = std::fwrite(&na, 4, 1, f) == 1;
    for (int l = 0; l < L && ok; l++) {
        const uint64_t len = t->len(l);
        ok = std::fwrite(&len, 8, 1, f) == 1;
    }
    ok = ok && std::fwrite(attrs, 4, L, f) == (size_t)L;
    for (int l = 0; l < L && ok; l++) ok = d[l].empty() || std::fwrite(d[l].data(), 4, d[l].size(), f) == d[l].size();
    for (int l = 0; l + 1 < L && ok; l++) ok = std::fwrite(o[l].data(), 8, o[l].size(), f) == o[l].size();
    if (std::fclose(f) != 0) ok = false;
    return ok ? AMJ_OK : fail(AMJ_EIO, std::string("trie_save_n: write failed for ") + path);
}

extern "C" int amj_trie_load_n(amj_ctx *ctx, const char *path, amj_trie **out, uint32_t *attrs, int *levels) {
    if (!ctx || !path || !out) return fail(AMJ_EINVAL, "trie_load_n: null argument");
    *out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(AMJ_EIO, std::string("trie_load_n: cannot open ") + path);
    uint32_t na = 0;
    uint64_t lens[TRIE_MAX_LEVELS] = {};
    uint32_t at[TRIE_MAX_LEVELS] = {};
    bool ok = std::fread(&na, 4, 1, f) == 1 && na >= 1 && na <= (uint32_t)TRIE_MAX_LEVELS &&
              std::fread(lens, 8, na, f) == na && std::fread(at, 4, na, f) == na;
    std::vector<std::vector<int32_t>> d(ok ? na : 0);
    std::vector<std::vector<uint64_t>> o(ok && na > 1 ? na - 1 : 0);
    for (uint32_t l = 0; ok && l < na; l++) {
        d[l].resize(lens[l]);
        ok = lens[l] == 0 || std::fread(d[l].data(), 4, lens[l], f) == lens[l];
    }
    for (uint32_t l = 0; ok && l + 1 < na; l++) {
        o[l].resize(lens[l] + 1);
        ok = std::fread(o[l].data(), 8, lens[l] + 1, f) == lens[l] + 1 && o[l][lens[l]] == lens[l + 1];
    }
    std::fclose(f);
    if (!ok) return fail(AMJ_EIO, "trie_load_n: bad, truncated or inconsistent file");
    auto *t = new amj_trie();
    t->ctx = ctx;
    t->tn.levels = (int)na;
    int rc = AMJ_OK;
    for (uint32_t l = 0; rc == AMJ_OK && l < na; l++) {
        t->tn.len[l] = lens[l];
        rc = t->tn.data[l].alloc(ctx, lens[l] ? lens[l] : 1);
        if (rc == AMJ_OK && lens[l] &&
            cudaMemcpyAsync(t->tn.data[l].p, d[l].data(), lens[l] * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
            rc = AMJ_ECUDA;
        if (rc == AMJ_OK && l + 1 < na) {
            rc = t->tn.off[l].alloc(ctx, lens[l] + 1);
            if (rc == AMJ_OK && cudaMemcpyAsync(t->tn.off[l].p, o[l].data(), (lens[l] + 1) * 8, cudaMemcpyHostToDevice,
                                                ctx->stream) != cudaSuccess)
                rc = AMJ_ECUDA;
        }
    }
    if (rc == AMJ_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = AMJ_ECUDA;
    if (rc != AMJ_OK) {
        (void)cudaGetLastError();
        delete t;
        return rc == AMJ_ECUDA ? fail(rc, "trie_load_n: device copy failed") : rc;
    }
    if (attrs)
        for (uint32_t l = 0; l < na; l++) attrs[l] = at[l];
    if (levels) *levels = (int)na;
    *out = t;
    return AMJ_OK;
}
