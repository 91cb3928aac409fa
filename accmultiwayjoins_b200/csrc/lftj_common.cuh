// Pieces of the leapfrog triejoin shared by the triangle (lftj.cu) and the
// 4-clique (lftj_clique4.cu) kernels: a device view of a 2-level trie, the
// child range of a value, and the warp-cooperative search and intersection of
// sorted arrays.
#pragma once
#include "amj_ops.cuh"

namespace amj {

struct TrieRef {
    const int32_t *data0;
    const uint64_t *off0;
    const int32_t *data1;
    const uint64_t *rowptr;
    uint64_t len0;
    uint64_t rp_count;
    int32_t rp_min;
};

inline TrieRef trie_ref(const Trie2 &t) {
    TrieRef r;
    r.data0 = t.data0.p;
    r.off0 = t.off0.p;
    r.data1 = t.data1.p;
    r.rowptr = t.rowptr.p;
    r.len0 = t.len0;
    r.rp_count = t.rp_count;
    r.rp_min = t.rp_min;
    return r;
}

__device__ __forceinline__ void child_range(const TrieRef &t, int32_t v, uint64_t &s, uint64_t &e) {
    if (t.rp_count) {
        const int64_t idx = (int64_t)v - (int64_t)t.rp_min;
        if (idx >= 0 && (uint64_t)idx < t.rp_count) {
            s = t.rowptr[idx];
            e = t.rowptr[idx + 1];
        } else {
            s = e = 0;
        }
        return;
    }
    uint64_t lo = 0, hi = t.len0;
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (t.data0[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    if (lo < t.len0 && t.data0[lo] == v) {
        s = t.off0[lo];
        e = t.off0[lo + 1];
    } else {
        s = e = 0;
    }
}

// first index in [lo, hi) whose value is >= target (hi if none); warp-uniform
// arguments, all lanes must call.  Exponential probe then 32-ary narrowing.
__device__ __forceinline__ uint64_t warp_lower_bound(const int32_t *A, uint64_t lo, uint64_t hi, int32_t target,
                                                     int lane) {
    if (lo >= hi) return hi;
    // exponential: lane l probes lo + 2^(l+5) - 1
    {
        const uint64_t off = lane < 27 ? ((uint64_t)32 << lane) - 1 : ~0ull;
        const uint64_t p = lo + off;
        const bool inr = off != ~0ull && p < hi;
        const bool less = inr && A[p] < target;
        const unsigned m = __ballot_sync(AMJ_FULL_MASK, less);
        const int c = __popc(m);   // probes 0..c-1 are below target
        const uint64_t nlo = c ? lo + ((uint64_t)32 << (c - 1)) : lo;
        const uint64_t q = lo + ((uint64_t)32 << c) - 1;   // first probe not below (or past the end)
        hi = (c < 27 && q < hi) ? q : hi;
        lo = nlo;
    }
    while (hi - lo > 32) {
        const uint64_t step = (hi - lo + 31) >> 5;
        const uint64_t p = lo + step * (uint64_t)(lane + 1) - 1;
        const bool inr = p < hi;
        const bool less = inr && A[p] < target;
        const int c = __popc(__ballot_sync(AMJ_FULL_MASK, less));
        const uint64_t q = lo + step * (uint64_t)(c + 1) - 1;
        lo = lo + step * (uint64_t)c;
        if (q < hi) hi = q;
    }
    const uint64_t p = lo + lane;
    const bool less = p < hi && A[p] < target;
    return lo + (uint64_t)__popc(__ballot_sync(AMJ_FULL_MASK, less));
}

// Warp-cooperative intersection of two strictly increasing arrays.  Every
// round (up to 32 values) calls round(match, value) on all lanes; the lanes
// with match hold the common values, in increasing lane order.  Warp-uniform
// arguments.
template <class Round>
__device__ __forceinline__ void warp_intersect_rounds(const int32_t *X, uint64_t nx, const int32_t *Y, uint64_t ny,
                                                      int lane, Round &&round) {
    const int32_t *B = X, *A = Y;
    uint64_t nb = nx, na = ny;
    if (nb > na) {
        B = Y; A = X;
        nb = ny; na = nx;
    }
    uint64_t i = 0, j = 0;
    while (i < nb && j < na) {
        const uint64_t bi = i + lane;
        const bool bval = bi < nb;
        const int32_t bv = bval ? B[bi] : 0;
        const uint32_t nvb = (nb - i) < 32 ? (uint32_t)(nb - i) : 32u;
        const int32_t bfirst = __shfl_sync(AMJ_FULL_MASK, bv, 0);
        const int32_t blast = __shfl_sync(AMJ_FULL_MASK, bv, nvb - 1);
        // gallop the haystack past values below the first needle
        {
            const uint64_t k = (j + 31 < na) ? j + 31 : na - 1;
            const int32_t a31 = A[k];
            if (a31 < bfirst) {
                if (k == na - 1) break;
                j = warp_lower_bound(A, j + 32, na, bfirst, lane);
                if (j >= na) break;
            }
        }
        const uint64_t aj = j + lane;
        const bool aval = aj < na;
        const int32_t av = aval ? A[aj] : 0;
        const uint32_t nva = (na - j) < 32 ? (uint32_t)(na - j) : 32u;
        const int32_t afirst = __shfl_sync(AMJ_FULL_MASK, av, 0);
        const int32_t alast = __shfl_sync(AMJ_FULL_MASK, av, nva - 1);
        // gallop the needles past values below the window
        if (blast < afirst) {
            i = warp_lower_bound(B, i + nvb, nb, afirst, lane);
            continue;
        }
        int pos = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            const int cand = pos + step;
            const int32_t v = __shfl_sync(AMJ_FULL_MASK, av, cand & 31);
            if ((uint32_t)cand < nva && v <= bv) pos = cand;
        }
        const int32_t at = __shfl_sync(AMJ_FULL_MASK, av, pos);
        const bool decided = bval && bv <= alast;
        round(decided && at == bv, bv);
        if (alast < blast) {
            i += __popc(__ballot_sync(AMJ_FULL_MASK, decided));
            j += nva;
        } else {
            i += nvb;
            j += __popc(__ballot_sync(AMJ_FULL_MASK, aval && av <= blast));
        }
    }
}

// The same, calling emit(value) on the lanes that hold a common value.
template <class Emit>
__device__ __forceinline__ void warp_intersect(const int32_t *X, uint64_t nx, const int32_t *Y, uint64_t ny, int lane,
                                               Emit &&emit) {
    warp_intersect_rounds(X, nx, Y, ny, lane, [&](bool m, int32_t v) {
        if (m) emit(v);
    });
}

// *out = max(*out, the longest child list among off[0..n])
static __global__ void max_children_kernel(const uint64_t *__restrict__ off, uint64_t n, unsigned long long *out) {
    unsigned long long m = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        m = (off[i + 1] - off[i] > m ? off[i + 1] - off[i] : m);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(AMJ_FULL_MASK, m, o);
        m = v > m ? v : m;
    }
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

}  // namespace amj
