// Kernels of the bucket-CSR build shared by its translation units.
#pragma once
#include "amj_ops.cuh"

namespace amj {

static __global__ void pack_key_rowid_kernel(const int32_t *__restrict__ key, uint64_t n, uint64_t *__restrict__ items) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        items[i] = ((uint64_t)(uint32_t)i << 32) | (uint32_t)key[i];
}

static __global__ void unpack_pairs_kernel(const uint64_t *__restrict__ items, uint64_t n, int32_t *__restrict__ lo,
                                    int32_t *__restrict__ hi) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t v = items[i];
        lo[i] = (int32_t)(uint32_t)v;
        if (hi) hi[i] = (int32_t)(uint32_t)(v >> 32);
    }
}

// bucket id of a sorted item
static __device__ __forceinline__ uint32_t item_bucket(uint64_t it, int key_mode, uint32_t mask) {
    uint32_t k = key_mode == KEY_PAIR ? hash_pair((int32_t)(uint32_t)it, (int32_t)(uint32_t)(it >> 32))
                                      : (uint32_t)it;
    return k & mask;
}

// counts[b] += run length of bucket b; items are sorted by bucket so equal
// buckets are contiguous: one atomic per run per warp.
static __global__ void bucket_hist_sorted_kernel(const uint64_t *__restrict__ items, uint64_t n, int key_mode,
                                          uint32_t mask, uint32_t *__restrict__ counts) {
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        const uint64_t i = base + lane;
        const bool valid = i < n;
        const uint32_t b = valid ? item_bucket(items[i], key_mode, mask) : 0xffffffffu;
        const uint32_t prev = __shfl_up_sync(AMJ_FULL_MASK, b, 1);
        const bool head = valid && (lane == 0 || prev != b);
        const unsigned heads = __ballot_sync(AMJ_FULL_MASK, head);
        const unsigned validm = __ballot_sync(AMJ_FULL_MASK, valid);
        if (head) {
            // run ends at the next head or at the last valid lane
            const unsigned after = heads & ~((2u << lane) - 1u);
            const int end = after ? __ffs(after) - 1 : 32 - __clz(validm);
            atomicAdd(&counts[b], (uint32_t)(end - lane));
        }
    }
}

}  // namespace amj
