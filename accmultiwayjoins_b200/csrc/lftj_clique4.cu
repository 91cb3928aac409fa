// ALFTJ 4-clique: the FOUR pattern A(0,1) B(1,2) C(2,3) D(0,3) E(0,2) F(1,3)
// (MHJ-GPU/exec_AMHJ.cu:50-69) as a leapfrog triejoin over one edge
// relation, attribute order a, b, c, d:
//   b in N(a);   c in N(a) ∩ N(b) = C(a,b);   d in C(a,b) ∩ N(c)
// where N(v) is v's child list in the relation's trie.  The reference's LFTJ
// stops at three attributes (LFTJ-GPU/config.h:16-17); this is its 4-attribute
// form for the FOUR query, the answer AMHJ FOUR gives on the same relation.
//
// Persistent warps claim 32 edges (a,b) at a time.
//  * An edge whose shorter list has at most 16 values is joined by its own
//    lane: C(a,b) by a merge into registers, then C(a,b) ∩ N(c) for every c
//    in it (merge, or per-value galloping search when N(c) is much longer).
//  * Longer edges are joined by the whole warp: C(a,b) by the warp
//    intersection, compacted with ballots into the warp's scratch area; then
//    the warp's lanes take 32 values c at a time, each intersecting C(a,b)
//    with N(c) on its own when the shorter side has at most 32 values, the
//    others one after another by the whole warp.
// Lists are strictly increasing (relations without duplicate edges, as for
// the triangle).
#include "lftj_common.cuh"

#include <algorithm>

namespace amj {

struct C4Args {
    const int32_t *src, *dst;   // the trie's level-1 entries: edge (src[j], dst[j])
    uint64_t n;
    TrieRef T;
    unsigned long long *cursor, *count, *checksum, *out_cursor;
    int32_t *out[4];
    uint64_t out_cap;
    int32_t *scratch;           // per warp: scratch_cap values
    uint64_t scratch_cap;
    int sorted_out;             // degree-ordered copy of an oriented relation: list tuples increasing
};

__device__ __forceinline__ uint64_t umin(uint64_t x, uint64_t y) { return x < y ? x : y; }
__device__ __forceinline__ uint64_t umax(uint64_t x, uint64_t y) { return x < y ? y : x; }

constexpr int C4_LANE_MAX = 16;   // shorter list of a lane-joined edge
constexpr int C4_LANE_PAIR = 32;  // shorter list of a lane-joined (C, N(c)) pair

// One 4-clique: count, checksum, and in write mode one output row.
template <bool WRITE>
__device__ __forceinline__ void c4_emit(const C4Args &A, int32_t a, int32_t b, int32_t c, int32_t d, uint64_t habc,
                                        unsigned long long &cnt, unsigned long long &chk) {
    cnt++;
    if (A.sorted_out) {
        // sorting network of four
        int32_t t;
        if (a > b) { t = a; a = b; b = t; }
        if (c > d) { t = c; c = d; d = t; }
        if (a > c) { t = a; a = c; c = t; }
        if (b > d) { t = b; b = d; d = t; }
        if (b > c) { t = b; b = c; c = t; }
        chk += amj_hash_step(amj_hash_step(amj_hash_step(amj_hash_step(AMJ_CHECKSUM_SEED, a), b), c), d);
    } else {
        chk += amj_hash_step(habc, d);
    }
    if (WRITE) {
        const unsigned long long p = atomicAdd(A.out_cursor, 1ull);
        if (p < A.out_cap) {
            A.out[0][p] = a;
            A.out[1][p] = b;
            A.out[2][p] = c;
            A.out[3][p] = d;
        }
    }
}

// Lane-local intersection of strictly increasing X[0,nx) and Y[0,ny): f(v)
// for each common value.  A merge when the lengths are close; otherwise every
// value of the shorter list is looked up in the longer one by galloping from
// the previous position.
template <class XP, class F>
__device__ __forceinline__ void lane_intersect(XP X, uint64_t nx, const int32_t *Y, uint64_t ny, F &&f) {
    if (nx == 0 || ny == 0) return;
    if (ny <= 8 * nx) {
        uint64_t p = 0, q = 0;
        while (p < nx && q < ny) {
            const int32_t x = X[p], y = Y[q];
            if (x == y) {
                f(x);
                p++;
                q++;
            } else if (x < y) {
                p++;
            } else {
                q++;
            }
        }
        return;
    }
    uint64_t q = 0;
    for (uint64_t p = 0; p < nx && q < ny; p++) {
        const int32_t x = X[p];
        // gallop: smallest q' >= q with Y[q'] >= x
        uint64_t step = 1, lo = q, hi = q;
        while (hi < ny && Y[hi] < x) {
            lo = hi + 1;
            hi = q + step;
            step <<= 1;
        }
        if (hi > ny) hi = ny;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (Y[mid] < x) lo = mid + 1;
            else hi = mid;
        }
        q = lo;
        if (q < ny && Y[q] == x) {
            f(x);
            q++;
        }
    }
}

template <bool WRITE>
__global__ __launch_bounds__(256) void lftj_clique4_kernel(const __grid_constant__ C4Args A) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    int32_t *buf = A.scratch + gw * A.scratch_cap;
    const int32_t *D1 = A.T.data1;
    unsigned long long cnt = 0, chk = 0;
    while (true) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(A.cursor, 32ull);
        base = __shfl_sync(AMJ_FULL_MASK, base, 0);
        if (base >= A.n) break;
        const uint64_t j = base + lane;
        const bool valid = j < A.n;
        int32_t a = 0, b = 0;
        uint64_t ta = 0, ea = 0, tb = 0, eb = 0;
        if (valid) {
            a = A.src[j];
            b = A.dst[j];
            child_range(A.T, a, ta, ea);
            if (ea > ta) child_range(A.T, b, tb, eb);
        }
        const uint64_t la = ea - ta, lb = eb - tb;
        const bool active = valid && la && lb;
        const bool small = active && umin(la, lb) <= (uint64_t)C4_LANE_MAX;
        const uint64_t hab = amj_hash_step(amj_hash_step(AMJ_CHECKSUM_SEED, a), b);
        // ---- short edges: one lane each
        if (small) {
            int32_t cl[C4_LANE_MAX];
            int m = 0;
            lane_intersect(D1 + (la <= lb ? ta : tb), umin(la, lb), D1 + (la <= lb ? tb : ta), umax(la, lb),
                           [&](int32_t v) { cl[m++] = v; });
            for (int i = 0; i < m; i++) {
                const int32_t c = cl[i];
                uint64_t tc, ec;
                child_range(A.T, c, tc, ec);
                const uint64_t habc = amj_hash_step(hab, c);
                lane_intersect(cl, (uint64_t)m, D1 + tc, ec - tc,
                               [&](int32_t d) { c4_emit<WRITE>(A, a, b, c, d, habc, cnt, chk); });
            }
        }
        // ---- long edges: the whole warp, one edge after another
        unsigned big = __ballot_sync(AMJ_FULL_MASK, active && !small);
        while (big) {
            const int l = __ffs(big) - 1;
            big &= big - 1;
            const int32_t wa = __shfl_sync(AMJ_FULL_MASK, a, l), wb = __shfl_sync(AMJ_FULL_MASK, b, l);
            const uint64_t wta = __shfl_sync(AMJ_FULL_MASK, ta, l), wea = __shfl_sync(AMJ_FULL_MASK, ea, l);
            const uint64_t wtb = __shfl_sync(AMJ_FULL_MASK, tb, l), web = __shfl_sync(AMJ_FULL_MASK, eb, l);
            const uint64_t whab = __shfl_sync(AMJ_FULL_MASK, hab, l);
            // C(a,b) into the scratch area (at most the shorter list, which fits it)
            uint64_t m = 0;
            warp_intersect_rounds(D1 + wta, wea - wta, D1 + wtb, web - wtb, lane, [&](bool hit, int32_t v) {
                const unsigned hm = __ballot_sync(AMJ_FULL_MASK, hit);
                if (hit) buf[m + __popc(hm & lt)] = v;
                m += __popc(hm);
            });
            __syncwarp();
            for (uint64_t i0 = 0; i0 < m; i0 += 32) {
                const uint64_t i = i0 + lane;
                const bool has = i < m;
                int32_t c = 0;
                uint64_t tc = 0, ec = 0;
                if (has) {
                    c = buf[i];
                    child_range(A.T, c, tc, ec);
                }
                const uint64_t lc = ec - tc;
                const uint64_t habc = amj_hash_step(whab, c);
                const bool pair = has && lc;
                const bool lone = pair && umin(lc, m) <= (uint64_t)C4_LANE_PAIR;
                if (lone) {
                    if (m <= lc) lane_intersect(buf, m, D1 + tc, lc,
                                                [&](int32_t d) { c4_emit<WRITE>(A, wa, wb, c, d, habc, cnt, chk); });
                    else lane_intersect(D1 + tc, lc, buf, m,
                                        [&](int32_t d) { c4_emit<WRITE>(A, wa, wb, c, d, habc, cnt, chk); });
                }
                unsigned wide = __ballot_sync(AMJ_FULL_MASK, pair && !lone);
                while (wide) {
                    const int l2 = __ffs(wide) - 1;
                    wide &= wide - 1;
                    const int32_t wc = __shfl_sync(AMJ_FULL_MASK, c, l2);
                    const uint64_t wtc = __shfl_sync(AMJ_FULL_MASK, tc, l2), wec = __shfl_sync(AMJ_FULL_MASK, ec, l2);
                    const uint64_t whabc = __shfl_sync(AMJ_FULL_MASK, habc, l2);
                    warp_intersect(buf, m, D1 + wtc, wec - wtc, lane,
                                   [&](int32_t d) { c4_emit<WRITE>(A, wa, wb, wc, d, whabc, cnt, chk); });
                }
            }
            __syncwarp();
        }
    }
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if (lane == 0 && cnt) {
        atomicAdd(A.count, cnt);
        atomicAdd(A.checksum, chk);
    }
}


struct C4Counters {
    unsigned long long cursor, count, checksum, out_cursor, max_deg;
};

// One 4-clique pass over the trie T of the edge relation: count and checksum,
// and the tuples when `out` is given (out_cap rows).
int lftj_clique4(amj_ctx *ctx, const Trie2 &T, int32_t *const *out, uint64_t out_cap, uint64_t *count,
                 uint64_t *checksum, uint64_t *written, double *kernel_ms, int sorted_out) {
    DBuf<C4Counters> ctr;
    AMJ_TRY(ctr.alloc(ctx, 1));
    AMJ_CUDA_TRY(cudaMemsetAsync(ctr.p, 0, sizeof(C4Counters), ctx->stream));
    *count = *checksum = 0;
    if (written) *written = 0;
    if (T.len1 == 0) return AMJ_OK;
    // the longest child list bounds C(a,b): the size of every warp's scratch area
    note_launch(ctx);
    max_children_kernel<<<(unsigned)std::min<uint64_t>((T.len0 + 255) / 256, (uint64_t)ctx->num_sms * 8), 256, 0,
                          ctx->stream>>>(T.off0.p, T.len0, &ctr.p->max_deg);
    AMJ_CUDA_TRY(cudaGetLastError());
    unsigned long long max_deg = 0;
    AMJ_CUDA_TRY(cudaMemcpyAsync(&max_deg, &ctr.p->max_deg, 8, cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    const bool write = out != nullptr;
    auto kern = write ? lftj_clique4_kernel<true> : lftj_clique4_kernel<false>;
    int per_sm = 0;
    AMJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0));
    uint64_t blocks = (uint64_t)ctx->num_sms * std::max(per_sm, 1);
    const uint64_t cap = std::max<unsigned long long>(max_deg, 1);
    // keep the scratch areas within 1/8 of the free device memory
    size_t fr = 0, tot = 0;
    AMJ_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    while (blocks > (uint64_t)ctx->num_sms && blocks * 8 * cap * 4 > fr / 8) blocks -= ctx->num_sms;
    if (blocks * 8 * cap * 4 > fr / 2) return fail(AMJ_ENOMEM, "LFTJ 4-clique: no room for the per-warp scratch");
    DBuf<int32_t> scratch;
    AMJ_TRY(scratch.alloc(ctx, blocks * 8 * cap));
    C4Args A{};
    A.src = T.src1.p;
    A.dst = T.data1.p;
    A.n = T.len1;
    A.T = trie_ref(T);
    A.cursor = &ctr.p->cursor;
    A.count = &ctr.p->count;
    A.checksum = &ctr.p->checksum;
    A.out_cursor = &ctr.p->out_cursor;
    if (write) {
        for (int i = 0; i < 4; i++) A.out[i] = out[i];
        A.out_cap = out_cap;
    }
    A.scratch = scratch.p;
    A.scratch_cap = cap;
    A.sorted_out = sorted_out;
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[0], ctx->stream));
    note_launch(ctx);
    kern<<<(unsigned)blocks, 256, 0, ctx->stream>>>(A);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[1], ctx->stream));
    C4Counters h;
    AMJ_CUDA_TRY(cudaMemcpyAsync(&h, ctr.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_TRY(status_check(ctx, "LFTJ 4-clique"));
    if (kernel_ms) *kernel_ms += event_ms(ctx->kev[0], ctx->kev[1]);
    *count = h.count;
    *checksum = h.checksum;
    if (written) *written = std::min<unsigned long long>(h.out_cursor, out_cap);
    return AMJ_OK;
}

}  // namespace amj
