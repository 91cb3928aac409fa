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
// ---- 4-cliques from triangle matrices (degree-ranked copy) ----
// Over the degree-ranked copy every 4-clique a < x < y < z (ranks) is a
// triangle (x, y, z) inside N+(a).  The wedge kernel in matrix mode records
// the triangles (a, x, y) as bits: row x - ta of a's matrix holds bit y - ta
// (ta = the start of T(a), so rows and columns are positions in N+(a)).
// Then the 4-cliques through (a, x, y) are the set bits of row x AND row y:
// persistent warps claim 32 level-1 entries (a, x) at a time, and for each
// one walk the bits y of row x; each AND is one word per lane (rows have at
// most 32 words: this path takes out-degrees up to 1024).  Found 4-cliques
// go to a per-warp queue of (entry lane, y, z) and are mapped to ids, sorted,
// hashed and written 32 at a time.
constexpr int C4M_THREADS = 256;
constexpr int C4M_WARPS = C4M_THREADS / 32;
constexpr int C4M_QCAP = 1024;   // queued 4-cliques per warp (ring; one step adds at most 1024)
constexpr uint32_t C4M_MAX_DEG = 1024;
// per warp: the queue, then the bits y of the current row x
constexpr size_t C4M_WARP_WORDS = C4M_QCAP + C4M_MAX_DEG / 2;
constexpr size_t C4M_SMEM = (size_t)C4M_WARPS * C4M_WARP_WORDS * 4;

struct C4MArgs {
    const int32_t *src1;     // rank a of every level-1 entry
    const int32_t *id1;      // vertex id of every level-1 value
    const int32_t *inv;      // rank -> vertex id
    const uint64_t *h1;      // first tuple-hash step of every vertex id
    TrieRef T;
    const uint64_t *moff;    // first matrix word of every rank
    const uint32_t *mtx;
    uint64_t n;
    unsigned long long *cursor, *count, *checksum, *out_cursor;
    int32_t *out[4];
    uint64_t out_cap;
};

template <bool WRITE>
__global__ __launch_bounds__(C4M_THREADS) void lftj_clique4_matrix_kernel(const __grid_constant__ C4MArgs A) {
    extern __shared__ uint32_t c4m_smem[];
    const int lane = threadIdx.x & 31;
    uint32_t *q = c4m_smem + (threadIdx.x >> 5) * C4M_WARP_WORDS;
    uint16_t *ylist = reinterpret_cast<uint16_t *>(q + C4M_QCAP);
    unsigned long long cnt = 0, chk = 0;
    uint32_t qh = 0, qn = 0;
    int32_t ida = 0, idx_ = 0;   // ids of this lane's entry (a, x)
    uint32_t ta32 = 0;           // start of T(a)
    // the first n queued 4-cliques, one per lane: (z << 15) | (y << 5) | lane of (a, x)
    auto flush = [&](uint32_t n) {
        __syncwarp();
        const bool mine = (uint32_t)lane < n;
        const uint32_t e = mine ? q[(qh + lane) & (C4M_QCAP - 1)] : 0u;
        const int l = (int)(e & 31u);
        const int32_t a = __shfl_sync(AMJ_FULL_MASK, ida, l);
        const int32_t x = __shfl_sync(AMJ_FULL_MASK, idx_, l);
        const uint32_t t0 = __shfl_sync(AMJ_FULL_MASK, ta32, l);
        __syncwarp();
        int32_t v[4] = {a, x, 0, 0};
        if (mine) {
            v[2] = A.id1[t0 + ((e >> 5) & 1023u)];
            v[3] = A.id1[t0 + (e >> 15)];
        }
        // the tuple in increasing order (sorting network of four)
        int32_t t;
        if (v[0] > v[1]) { t = v[0]; v[0] = v[1]; v[1] = t; }
        if (v[2] > v[3]) { t = v[2]; v[2] = v[3]; v[3] = t; }
        if (v[0] > v[2]) { t = v[0]; v[0] = v[2]; v[2] = t; }
        if (v[1] > v[3]) { t = v[1]; v[1] = v[3]; v[3] = t; }
        if (v[1] > v[2]) { t = v[1]; v[1] = v[2]; v[2] = t; }
        if (WRITE) {
            unsigned long long at = 0;
            if (lane == 0) at = atomicAdd(A.out_cursor, (unsigned long long)n);
            at = __shfl_sync(AMJ_FULL_MASK, at, 0);
            if (mine && at + lane < A.out_cap)
                for (int i = 0; i < 4; i++) A.out[i][at + lane] = v[i];
        }
        if (mine) {
            cnt++;
            // the first step from the per-id table: one load instead of a mix
            chk += amj_hash_step(amj_hash_step(amj_hash_step(A.h1[v[0]], v[1]), v[2]), v[3]);
        }
        qh = (qh + n) & (C4M_QCAP - 1);
        qn -= n;
    };
    while (true) {
        unsigned long long at = 0;
        if (lane == 0) at = atomicAdd(A.cursor, 32ull);
        at = __shfl_sync(AMJ_FULL_MASK, at, 0);
        if (at >= A.n) break;
        const uint64_t j = at + lane;
        const bool valid = j < A.n;
        uint32_t w = 0;
        uint64_t rowbase = 0, mbase = 0;
        if (valid) {
            const int32_t a = A.src1[j];
            uint64_t ta, te;
            child_range(A.T, a, ta, te);
            w = (uint32_t)((te - ta + 31) / 32);
            mbase = A.moff[a];
            rowbase = mbase + (j - ta) * w;
            ida = A.inv[a];
            idx_ = A.id1[j];
            ta32 = (uint32_t)ta;
        }
        unsigned todo = __ballot_sync(AMJ_FULL_MASK, valid && w > 0);
        while (todo) {
            const int l = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t wl = __shfl_sync(AMJ_FULL_MASK, w, l);
            const uint64_t rb = __shfl_sync(AMJ_FULL_MASK, rowbase, l);
            const uint64_t mb = __shfl_sync(AMJ_FULL_MASK, mbase, l);
            // row x, one word per lane; its bits y are the triangles (a, x, y)
            const uint32_t rx = (uint32_t)lane < wl ? A.mtx[rb + lane] : 0u;
            const uint32_t nyl = __popc(rx);
            const uint32_t yincl = warp_inclusive_scan(nyl, lane);
            const uint32_t ny = __shfl_sync(AMJ_FULL_MASK, yincl, 31);
            if (ny == 0) continue;
            {
                uint32_t p = yincl - nyl, m = rx;
                while (m) {
                    const uint32_t b = __ffs(m) - 1;
                    m &= m - 1;
                    ylist[p++] = (uint16_t)(lane * 32 + b);
                }
            }
            __syncwarp();
            // 32 / wp bits y per step, wp lanes (one per word of row y) each
            uint32_t wp = 1;
            while (wp < wl) wp <<= 1;
            const uint32_t G = 32 / wp, slot = (uint32_t)lane / wp, wd = (uint32_t)lane & (wp - 1);
            const uint32_t rxw = __shfl_sync(AMJ_FULL_MASK, rx, (int)wd);
            for (uint32_t b0 = 0; b0 < ny; b0 += G) {
                const uint32_t yi = b0 + slot;
                uint32_t c = 0, y = 0;
                if (yi < ny) {
                    y = ylist[yi];
                    // z: bits of row x AND row y (row y holds bits above y only)
                    if (wd < wl && wd >= y / 32) c = rxw & A.mtx[mb + (uint64_t)y * wl + wd];
                }
                const uint32_t nh = __popc(c);
                const uint32_t incl = warp_inclusive_scan(nh, lane);
                const uint32_t tot = __shfl_sync(AMJ_FULL_MASK, incl, 31);
                if (tot) {
                    if (qn + tot > C4M_QCAP) flush(qn);   // make room (tot is at most 1024)
                    uint32_t pos = qh + qn + incl - nh;
                    while (c) {
                        const uint32_t bz = __ffs(c) - 1;
                        c &= c - 1;
                        q[pos++ & (C4M_QCAP - 1)] = ((wd * 32 + bz) << 15) | (y << 5) | (uint32_t)l;
                    }
                    qn += tot;
                    while (qn >= 32) flush(32);
                }
            }
            __syncwarp();
        }
        if (qn) flush(qn);
    }
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd(A.count, cnt);
        atomicAdd(A.checksum, chk);
    }
}

__global__ void level1_ids_kernel(const int32_t *__restrict__ data1, uint64_t n, const int32_t *__restrict__ inv,
                                  int32_t *__restrict__ id1) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        id1[i] = inv[data1[i]];
}

int lftj_tri_matrices(amj_ctx *ctx, const Trie2 &R, const uint64_t *wedge, uint64_t nv, uint32_t rank_bits,
                      uint64_t max_words, DBuf<uint64_t> *moff, uint32_t **mtx, uint64_t *words);

// Largest child list of the trie (its longest out-neighbour list).
static int trie_max_children(amj_ctx *ctx, const Trie2 &T, uint64_t *maxc) {
    *maxc = 0;
    if (T.len0 == 0) return AMJ_OK;
    DBuf<unsigned long long> m;
    AMJ_TRY(m.alloc(ctx, 1));
    AMJ_CUDA_TRY(cudaMemsetAsync(m.p, 0, sizeof(unsigned long long), ctx->stream));
    note_launch(ctx);
    max_children_kernel<<<(unsigned)std::min<uint64_t>((T.len0 + 255) / 256, (uint64_t)ctx->num_sms * 8), 256, 0,
                          ctx->stream>>>(T.off0.p, T.len0, m.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    unsigned long long h = 0;
    AMJ_CUDA_TRY(cudaMemcpyAsync(&h, m.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    *maxc = h;
    return AMJ_OK;
}

// Prepared state of the matrix path over one degree-ranked trie.
struct C4Matrix {
    DBuf<uint64_t> moff;
    uint32_t *mtx = nullptr;   // the context's matrix buffer
    DBuf<int32_t> id1;
    DBuf<uint64_t> h1;         // amj_hash_step(AMJ_CHECKSUM_SEED, id) of every vertex id
};

// the first step of the tuple hash of every vertex id in [0, nv)
__global__ void id_hash_kernel(uint64_t nv, uint64_t *__restrict__ h1) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nv; i += (uint64_t)gridDim.x * blockDim.x)
        h1[i] = amj_hash_step(AMJ_CHECKSUM_SEED, (int32_t)i);
}

// Whether the matrix path takes the degree-ranked trie T (every out-degree at
// most 1024, the matrices within half the free device memory), and if so the
// triangle matrices and the ids of level 1.
int lftj_clique4_matrix_prepare(amj_ctx *ctx, const Trie2 &T, const int32_t *inv, const uint64_t *wedge, uint64_t nv,
                                uint32_t rank_bits, C4Matrix **out) {
    *out = nullptr;
    uint64_t maxc = 0;
    AMJ_TRY(trie_max_children(ctx, T, &maxc));
    if (maxc > C4M_MAX_DEG) return AMJ_OK;
    size_t fr = 0, tot = 0;
    AMJ_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    auto *m = new C4Matrix();
    uint64_t words = 0;
    // at most half the free memory, or the buffer the context already holds
    const uint64_t max_words = std::max<uint64_t>(fr / 2 / 4, ctx->c4_mtx_words);
    int rc = lftj_tri_matrices(ctx, T, wedge, nv, rank_bits, max_words, &m->moff, &m->mtx, &words);
    if (rc == AMJ_ENOMEM) {   // the matrices do not fit: not this path
        delete m;
        return AMJ_OK;
    }
    if (rc == AMJ_OK) rc = m->id1.alloc(ctx, T.len1 ? T.len1 : 1);
    if (rc == AMJ_OK && T.len1) {
        note_launch(ctx);
        level1_ids_kernel<<<(unsigned)std::min<uint64_t>((T.len1 + 255) / 256, (uint64_t)ctx->num_sms * 16), 256, 0,
                            ctx->stream>>>(T.data1.p, T.len1, inv, m->id1.p);
        if (cudaGetLastError() != cudaSuccess) rc = fail(AMJ_ECUDA, "LFTJ 4-clique: level-1 ids");
    }
    // vertex ids are the ranks' images, all below nv
    if (rc == AMJ_OK) rc = m->h1.alloc(ctx, nv ? nv : 1);
    if (rc == AMJ_OK && nv) {
        note_launch(ctx);
        id_hash_kernel<<<(unsigned)std::min<uint64_t>((nv + 255) / 256, (uint64_t)ctx->num_sms * 16), 256, 0,
                         ctx->stream>>>(nv, m->h1.p);
        if (cudaGetLastError() != cudaSuccess) rc = fail(AMJ_ECUDA, "LFTJ 4-clique: id hashes");
    }
    if (rc != AMJ_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return AMJ_OK;
}

void lftj_clique4_matrix_release(C4Matrix *m) { delete m; }

// 4-cliques of the degree-ranked trie T from its prepared matrices: count and
// checksum, and with out the sorted tuples (out_cap rows available).
int lftj_clique4_matrix(amj_ctx *ctx, const Trie2 &T, const int32_t *inv, const C4Matrix *m, int32_t *const *out,
                        uint64_t out_cap, uint64_t *count, uint64_t *checksum, uint64_t *written, double *kernel_ms) {
    DBuf<C4Counters> ctr;
    AMJ_TRY(ctr.alloc(ctx, 1));
    AMJ_CUDA_TRY(cudaMemsetAsync(ctr.p, 0, sizeof(C4Counters), ctx->stream));
    *count = *checksum = 0;
    if (written) *written = 0;
    if (T.len1 == 0) return AMJ_OK;
    const bool write = out != nullptr;
    C4MArgs A{};
    A.src1 = T.src1.p;
    A.id1 = m->id1.p;
    A.inv = inv;
    A.h1 = m->h1.p;
    A.T = trie_ref(T);
    A.moff = m->moff.p;
    A.mtx = m->mtx;
    A.n = T.len1;
    A.cursor = &ctr.p->cursor;
    A.count = &ctr.p->count;
    A.checksum = &ctr.p->checksum;
    A.out_cursor = &ctr.p->out_cursor;
    if (write) {
        for (int i = 0; i < 4; i++) A.out[i] = out[i];
        A.out_cap = out_cap;
    }
    auto kern = write ? lftj_clique4_matrix_kernel<true> : lftj_clique4_matrix_kernel<false>;
    AMJ_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C4M_SMEM));
    int per_sm = 0;
    AMJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C4M_THREADS, C4M_SMEM));
    if (per_sm < 1) per_sm = 1;
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[0], ctx->stream));
    note_launch(ctx);
    kern<<<(unsigned)(ctx->num_sms * per_sm), C4M_THREADS, C4M_SMEM, ctx->stream>>>(A);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[1], ctx->stream));
    C4Counters h;
    AMJ_CUDA_TRY(cudaMemcpyAsync(&h, ctr.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (kernel_ms) *kernel_ms += event_ms(ctx->kev[0], ctx->kev[1]);
    *count = h.count;
    *checksum = h.checksum;
    if (written) *written = std::min<unsigned long long>(h.out_cursor, out_cap);
    return AMJ_OK;
}

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
