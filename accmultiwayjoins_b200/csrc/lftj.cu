// ALFTJ: leapfrog triejoin over 2-level tries, DFS and BFS.
//
// Query shape: the triangle R(a,b) S(b,c) T(a,c) with attribute order a,b,c,
// as a self-join over one edge relation (LFTJ-GPU/exec_LFTJ.cu:96-102,
// 218-222) or over three relations whose attributes form that pattern.
//
// DFS (reference ALFTJ_count / ALFTJ_write, LFTJ-GPU/ALFTJ.cuh:213-1043):
// level a is the level-0 array of R (= T's), level b the children of a in R
// (the level-1 entries of R, walked edge by edge), level c the intersection
// of S's children of b with T's children of a.  Persistent warps claim 32
// level-1 entries of R at a time.  Per entry the two child ranges are found
// with one dense row-pointer load each (or a binary search of level 0).
// Short pairs are intersected by the owning lane with a sequential merge;
// long pairs by the whole warp: 32 needles of the shorter list against a
// 32-wide window of the longer one, membership by a shuffle binary search,
// and ballot-driven galloping (exponential then 32-ary search) over runs that
// cannot match.  Counting and the tuple checksum happen in registers; in
// write mode each warp reserves output rows with one atomic per round.
// Over one oriented edge relation with ws=1 the degree-ranked copy is joined
// instead, by the wedge kernel below: for every edge (a, b), the values of
// T(a) after b are tested against a per-warp bitmap of S(b).
//
// BFS (reference LFTJ_BFS np_join_np / p_join_np / p_join_p,
// LFTJ-GPU/LFTJ_BFS.cuh:143-500): level-synchronous.  One kernel counts the
// candidates of every (a,b) entry (the shorter of its two child lists), a
// scan turns the counts into candidate offsets, and a load-balanced kernel
// gives every thread one candidate c: the owning entry is found by a
// shared-memory binary search over the tile's offsets, then c is looked up in
// the other child list.  Everything runs on the device, including the load
// balancing the reference does on the CPU (LFTJ_BFS.cuh:396-397), and the
// count it computes is returned (the reference returns 0, :496).  Over the
// degree-ranked copy of one relation the candidates of (a,b) are T(a)'s
// values after b, searched in S(b).
#include "lftj_common.cuh"

#include <algorithm>

namespace amj {

struct TriArgs {
    const int32_t *r_src;   // level-0 value of every level-1 entry of R (a)
    const int32_t *r_dst;   // level-1 values of R (b)
    uint64_t r_n;
    TrieRef S, T;
    unsigned long long *cursor;
    unsigned long long *count;
    unsigned long long *checksum;
    unsigned long long *out_cursor;
    int32_t *out[3];
    uint64_t out_cap;
    int small_sum;   // merge by one lane when |X|+|Y| <= small_sum
    // heavy vertices (bitmap kernel): R's level-0 entries with at least
    // heavy_deg children whose T-children span at most bitmap_bits values
    TrieRef R;
    uint64_t r_lo, r_hi;          // R level-1 slice handled by this launch
    unsigned long long *cursor0;  // claim cursor of the bitmap kernel over heavy_list
    const uint32_t *heavy_list;   // R's level-0 indexes of the heavy vertices
    const unsigned long long *heavy_n;
    uint32_t heavy_deg;           // 0: no bitmap kernel
    uint32_t bitmap_bits;
    int sorted_out;               // the tries hold a degree-ordered copy of an oriented relation:
                                  // every triangle is listed with its values in increasing order
    // wedge kernel: the tries hold the degree-ranked copy (vertex = rank in
    // (degree, id) order); inv[rank] is the vertex id
    const int32_t *inv;
    const uint64_t *wedge;        // (b << 32 | entry) of this slice's entries, sorted by b
    const uint64_t *moff;         // matrix mode: first word of every vertex a's matrix
    uint32_t *mtx;                // matrix mode: row x of a's matrix has bit y when (a, x, y) is a triangle
    const int32_t *src1;          // level-0 value of every level-1 entry of R
    uint32_t rank_base;           // first rank of the per-warp bitmap
    uint32_t rank_bits;           // ranks the bitmap covers
    unsigned long long *cursor_r; // claim cursor of the wedge kernel
    int bfs_wedge;                // BFS over one degree-ordered relation (R = S = T): the
                                  // candidates of entry (a, b) are T(a)'s values after b
    const struct RankId *hid;     // wedge kernel: id and first hash step of every rank
};

// The vertex id of a rank and the first step of the tuple hash over it,
// amj_hash_step(AMJ_CHECKSUM_SEED, id): one 16-byte load gives a hit's id
// and, when that id is the triangle's smallest, its hash prefix.
struct __align__(16) RankId {
    int32_t id;
    uint32_t pad;
    uint64_t h1;
};

__global__ void rank_ids_kernel(const int32_t *__restrict__ inv, uint64_t nv, RankId *__restrict__ hid) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nv; i += (uint64_t)gridDim.x * blockDim.x) {
        const int32_t id = inv[i];
        hid[i] = RankId{id, 0u, amj_hash_step(AMJ_CHECKSUM_SEED, id)};
    }
}

// A triangle found as (a, b, c) in the tuple the query lists: attribute order,
// or increasing order for a degree-ordered copy of an oriented relation
// (whose triangles, in attribute order, are exactly the increasing triples).
__device__ __forceinline__ void tri_order(const TriArgs &A, int32_t &a, int32_t &b, int32_t &c) {
    if (!A.sorted_out) return;
    int32_t t;
    if (a > b) { t = a; a = b; b = t; }
    if (b > c) { t = b; b = c; c = t; }
    if (a > b) { t = a; a = b; b = t; }
}

// checksum term of the triangle (a, b, c); hab is the hash of (a, b)
__device__ __forceinline__ uint64_t tri_chk(const TriArgs &A, uint64_t hab, int32_t a, int32_t b, int32_t c) {
    if (!A.sorted_out) return amj_hash_step(hab, c);
    tri_order(A, a, b, c);
    return amj_hash_step(amj_hash_step(amj_hash_step(AMJ_CHECKSUM_SEED, a), b), c);
}

// checksum term of the triangle (a, b, c) from scratch
__device__ __forceinline__ uint64_t tri_chk3(const TriArgs &A, int32_t a, int32_t b, int32_t c) {
    tri_order(A, a, b, c);
    return amj_hash_step(amj_hash_step(amj_hash_step(AMJ_CHECKSUM_SEED, a), b), c);
}

__device__ __forceinline__ void tri_store(const TriArgs &A, unsigned long long p, int32_t a, int32_t b, int32_t c) {
    tri_order(A, a, b, c);
    A.out[0][p] = a;
    A.out[1][p] = b;
    A.out[2][p] = c;
}

// A level-0 value a of R is "heavy" when it has at least heavy_deg children in
// R and its children in T span at most bitmap_bits values: its edges are
// then joined by the bitmap kernel, all others by the warp kernel.
__device__ __forceinline__ bool heavy_vertex(const TriArgs &A, uint64_t r_deg, uint64_t ta, uint64_t ea,
                                             int32_t &lo, uint32_t &span) {
    if (A.heavy_deg == 0 || r_deg < A.heavy_deg || ea <= ta) return false;
    lo = A.T.data1[ta];
    const int64_t sp = (int64_t)A.T.data1[ea - 1] - (int64_t)lo + 1;
    span = (uint32_t)sp;
    return sp > 0 && sp <= (int64_t)A.bitmap_bits;
}

// R's level-0 indexes of the vertices the bitmap kernel owns, in any order
__global__ void heavy_list_kernel(const __grid_constant__ TriArgs A, uint32_t *list, unsigned long long *n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < A.R.len0;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t rs = A.R.off0[i], re = A.R.off0[i + 1];
        if ((rs > A.r_lo ? rs : A.r_lo) >= (re < A.r_hi ? re : A.r_hi)) continue;
        uint64_t ta, ea;
        child_range(A.T, A.R.data0[i], ta, ea);
        int32_t lo;
        uint32_t span;
        if (heavy_vertex(A, re - rs, ta, ea, lo, span)) list[atomicAdd(n, 1ull)] = (uint32_t)i;
    }
}

constexpr int BM_THREADS = 1024;
constexpr int BM_UNROLL = 8;
constexpr uint32_t BM_SEG = 1024;   // values of one child list per warp work item

// Bitmap kernel: one block per heavy vertex a at a time.  The children of a
// in T are set in a shared-memory bitmap (one bit per value in their span,
// up to 2^20 values = 128 KB); then the children lists of every b in a's
// R-children are streamed through the block, 1024 edges per batch, with a
// block scan over their lengths so every thread takes one candidate c per
// step (load-balanced, coalesced) and tests bit c.  Each child list is read
// once per (a,b) and tested with one shared-memory load, instead of a
// galloping search per needle window.
template <bool WRITE>
__global__ __launch_bounds__(BM_THREADS, 1) void lftj_tri_bitmap_kernel(const __grid_constant__ TriArgs A) {
    extern __shared__ __align__(16) unsigned char bm_smem[];
    const uint32_t words = (A.bitmap_bits + 31) / 32;
    uint32_t *bits = (uint32_t *)bm_smem;
    unsigned long long *pre = (unsigned long long *)(bm_smem + (size_t)words * 4);  // inclusive
    unsigned long long *hab = pre + BM_THREADS;
    uint32_t *sbeg = (uint32_t *)(hab + BM_THREADS);
    int32_t *bval = (int32_t *)(sbeg + BM_THREADS);
    uint32_t *segpre = (uint32_t *)(bval + BM_THREADS);
    __shared__ unsigned long long s_i;
    __shared__ unsigned long long s_wsum[BM_THREADS / 32 + 1];
    __shared__ uint32_t s_next;
    __shared__ uint32_t s_ssum[BM_THREADS / 32 + 1];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t w = tid; w < words; w += BM_THREADS) bits[w] = 0u;
    unsigned long long cnt = 0, chk = 0;
    __syncthreads();
    while (true) {
        if (tid == 0) {
            const unsigned long long x = atomicAdd(A.cursor0, 1ull);
            s_i = x < *A.heavy_n ? A.heavy_list[x] : ~0ull;
        }
        __syncthreads();
        const unsigned long long i = s_i;
        __syncthreads();
        if (i >= A.R.len0) break;
        const uint64_t rs = A.R.off0[i], re = A.R.off0[i + 1];
        const uint64_t es = rs > A.r_lo ? rs : A.r_lo, ee = re < A.r_hi ? re : A.r_hi;
        if (es >= ee) continue;
        const int32_t a = A.R.data0[i];
        uint64_t ta, ea;
        child_range(A.T, a, ta, ea);
        int32_t lo = 0;
        uint32_t span = 0;
        if (!heavy_vertex(A, re - rs, ta, ea, lo, span)) continue;
        for (uint64_t k = ta + tid; k < ea; k += BM_THREADS) {
            const uint32_t r = (uint32_t)(A.T.data1[k] - lo);
            atomicOr(&bits[r >> 5], 1u << (r & 31));
        }
        const uint64_t ha = amj_hash_step(AMJ_CHECKSUM_SEED, a);
        __syncthreads();
        for (uint64_t bs = es; bs < ee; bs += BM_THREADS) {
            const uint64_t j = bs + tid;
            unsigned long long len = 0;
            uint64_t sb = 0, eb = 0;
            int32_t b = 0;
            if (j < ee) {
                b = A.R.data1[j];
                child_range(A.S, b, sb, eb);
                len = eb - sb;
            }
            // block inclusive scans of len and of the list's segment count
            const uint32_t nseg = (uint32_t)((len + BM_SEG - 1) / BM_SEG);
            unsigned long long incl = warp_inclusive_scan(len, lane);
            uint32_t sincl = warp_inclusive_scan(nseg, lane);
            if (lane == 31) {
                s_wsum[warp] = incl;
                s_ssum[warp] = sincl;
            }
            __syncthreads();
            if (warp == 0) {
                unsigned long long w = lane < BM_THREADS / 32 ? s_wsum[lane] : 0ull;
                unsigned long long wi = warp_inclusive_scan(w, lane);
                s_wsum[lane] = wi - w;
                uint32_t sw = lane < BM_THREADS / 32 ? s_ssum[lane] : 0u;
                uint32_t swi = warp_inclusive_scan(sw, lane);
                s_ssum[lane] = swi - sw;
                if (lane == 31) s_ssum[BM_THREADS / 32] = swi;
            }
            __syncthreads();
            pre[tid] = s_wsum[warp] + incl;
            segpre[tid] = s_ssum[warp] + sincl;
            sbeg[tid] = (uint32_t)sb;
            hab[tid] = amj_hash_step(ha, b);
            bval[tid] = b;
            const uint32_t total_seg = s_ssum[BM_THREADS / 32];
            const uint32_t nb = (uint32_t)((ee - bs) < BM_THREADS ? (ee - bs) : BM_THREADS);
            if (tid == 0) s_next = 0;
            __syncthreads();
            // warps claim segments of at most BM_SEG values of the child lists
            // (balanced across warps whatever the list lengths) and stream each,
            // 32 x BM_UNROLL values per step with all loads in flight before the tests
            while (true) {
                uint32_t sg = 0;
                if (lane == 0) sg = atomicAdd(&s_next, 1u);
                sg = __shfl_sync(AMJ_FULL_MASK, sg, 0);
                if (sg >= total_seg) break;
                uint32_t slo = 0, shi = nb - 1;
                while (slo < shi) {
                    const uint32_t mid = (slo + shi) >> 1;
                    if (segpre[mid] > sg) shi = mid;
                    else slo = mid + 1;
                }
                const uint32_t li = slo;
                const uint32_t first_seg = li ? segpre[li - 1] : 0u;
                const unsigned long long lbeg = li ? pre[li - 1] : 0ull;
                const uint32_t llen = (uint32_t)(pre[li] - lbeg);
                const uint32_t kbeg = (sg - first_seg) * BM_SEG;
                const uint32_t len = (llen - kbeg) < BM_SEG ? (llen - kbeg) : BM_SEG;
                const int32_t *lst = A.S.data1 + sbeg[li] + kbeg;
                const uint64_t hb = hab[li];
                // value c of the list is a hit when lo <= c < lo + span and its bit is set
                auto test = [&](int32_t c) -> bool {
                    const uint32_t r = (uint32_t)c - (uint32_t)lo;
                    return c >= lo && r < span && ((bits[r >> 5] >> (r & 31)) & 1u);
                };
                auto emit = [&](bool hit, int32_t c) {
                    if (!WRITE) {
                        if (hit) {
                            cnt++;
                            chk += tri_chk(A, hb, a, bval[li], c);
                        }
                    } else {
                        const unsigned m = __ballot_sync(AMJ_FULL_MASK, hit);
                        if (m) {
                            unsigned long long base = 0;
                            if (lane == 0) base = atomicAdd(A.out_cursor, (unsigned long long)__popc(m));
                            base = __shfl_sync(AMJ_FULL_MASK, base, 0);
                            if (hit) {
                                cnt++;
                                chk += tri_chk(A, hb, a, bval[li], c);
                                const unsigned long long p = base + __popc(m & lanemask_lt());
                                if (p < A.out_cap) tri_store(A, p, a, bval[li], c);
                            }
                        }
                    }
                };
                uint32_t k0 = 0;
                // full blocks of 32 x BM_UNROLL values: all loads issued before the tests
                for (; k0 + 32 * BM_UNROLL <= len; k0 += 32 * BM_UNROLL) {
                    int32_t cv[BM_UNROLL];
#pragma unroll
                    for (int u = 0; u < BM_UNROLL; u++) cv[u] = lst[k0 + u * 32 + lane];
#pragma unroll
                    for (int u = 0; u < BM_UNROLL; u++) emit(test(cv[u]), cv[u]);
                }
                // the rest (all of a short list) 32 values at a time
                for (; k0 < len; k0 += 32) {
                    const uint32_t k = k0 + lane;
                    const bool in = k < len;
                    const int32_t c = in ? lst[k] : 0;
                    emit(in && test(c), c);
                }
            }
            __syncthreads();
        }
        for (uint64_t k = ta + tid; k < ea; k += BM_THREADS) {
            const uint32_t r = (uint32_t)(A.T.data1[k] - lo);
            bits[r >> 5] = 0u;
        }
        __syncthreads();
    }
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if (lane == 0 && cnt) {
        atomicAdd(A.count, cnt);
        atomicAdd(A.checksum, chk);
    }
}

// ---- wedge kernel ----
// The degree-ranked copy of an oriented edge relation: every vertex renamed
// to its rank in (degree, id) order, edges from the lower to the higher
// rank.  A triangle is then a wedge a -> b, a -> c with b < c closed by the
// edge b -> c: for every edge (a, b), the children of a ranked above b (the
// suffix of T(a) after b) are tested against the children of b.  That is
// sum over a of C(d+(a), 2) tests (1.23 G on R-MAT scale 20, against 4.42 G
// for streaming S(b) per edge).  The edges come grouped by b (a stable sort
// of (b, entry)), so each warp keeps the children of one b as a bitmap in
// shared memory.  Out-neighbours concentrate on the highest ranks (on R-MAT
// scale 20, 99.8% of the tested values lie in the top 32K ranks), so the
// bitmap covers the top rank_bits ranks (4 KB) and a test is one
// shared-memory load; the rare values below it are binary-searched in
// S(b)'s low prefix (a sorted prefix, kept in shared memory up to 256).
// Persistent warps claim 32 edges at a time; each edge's suffix streams
// through the warp in aligned 16-byte quads.  Hits go to a per-warp queue
// of (c, edge) pairs; the id mapping, the checksum and the writes run on 32
// queued triangles at a time, so lanes without a hit do not wait on them.
// Per edge the lane keeps the ids of a and b in increasing order (lo, hi)
// and the hash prefix of lo; per hit one 16-byte load gives c's id and its
// own prefix, so a triangle costs two hash steps: the tuple is (min(c, lo),
// median, max(c, hi)) and its first step is the prefix of c or of lo.
// The queue packs a hit into 32 bits (rank << 5 | lane) when every rank is
// below 2^27; wider ranks take 64-bit entries.  Three blocks run per SM: the
// kernel is bound by the integer (ALU) pipe, and a fourth block, which needs
// at most 64 registers a thread, made it slower (3.85 against 3.63 ms at
// R-MAT scale 20).
constexpr int TR_THREADS = 256;
constexpr int TR_WARPS = TR_THREADS / 32;
constexpr uint32_t TR_BITS = 32768;            // bitmap ranks per warp (the most)
constexpr int TR_LOWCAP = 192;                 // low prefix entries kept in shared memory
constexpr int TR_UNROLL = 4;                   // quads per lane per step
constexpr int TR_QCAP = 512;                   // queued hits per warp (ring)
constexpr uint64_t TR_NARROW_RANKS = 1ull << 27;

template <bool WIDE>
struct TrWarp {
    uint32_t bm[TR_BITS / 32];
    int32_t low[TR_LOWCAP];
    uint32_t q[TR_QCAP * (WIDE ? 2 : 1)];   // narrow: rank << 5 | lane; wide: (rank, lane) pairs
};
template <bool WIDE>
constexpr size_t tr_smem() { return TR_WARPS * sizeof(TrWarp<WIDE>); }
static_assert(sizeof(TrWarp<false>) % 16 == 0 && sizeof(TrWarp<true>) % 16 == 0, "TrWarp keeps 16-byte alignment");
static_assert(TR_QCAP >= 32 * 4 * TR_UNROLL, "the queue takes one step's hits");

template <bool WIDE>
__device__ __forceinline__ void tr_qput(TrWarp<WIDE> &W, uint32_t pos, int32_t c, int lane) {
    pos &= TR_QCAP - 1;
    if (WIDE) {
        W.q[2 * pos] = (uint32_t)c;
        W.q[2 * pos + 1] = (uint32_t)lane;
    } else {
        W.q[pos] = ((uint32_t)c << 5) | (uint32_t)lane;
    }
}
template <bool WIDE>
__device__ __forceinline__ void tr_qget(const TrWarp<WIDE> &W, uint32_t pos, int32_t &c, int &lane) {
    pos &= TR_QCAP - 1;
    if (WIDE) {
        c = (int32_t)W.q[2 * pos];
        lane = (int)W.q[2 * pos + 1];
    } else {
        const uint32_t e = W.q[pos];
        c = (int32_t)(e >> 5);
        lane = (int)(e & 31u);
    }
}

__device__ __forceinline__ bool tr_sorted_find(const int32_t *v, uint64_t n, int32_t c) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (v[mid] < c) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && v[lo] == c;
}

// bit of rank value c in the warp's bitmap (the index stays in bounds for
// values outside it, which the caller masks off)
__device__ __forceinline__ uint32_t tr_bit(const uint32_t *bm, int32_t c, uint32_t base) {
    const uint32_t r = ((uint32_t)c - base) & (TR_BITS - 1);
    return __funnelshift_r(bm[r >> 5], 0u, r) & 1u;
}

// MODE 0: count and checksum; 1: also write the tuples; 2 (matrix mode):
// record every triangle (a, x, y) as bit y - ta of row x - ta of a's matrix
// (ta = the start of T(a) in level 1; rows have ceil(d+(a) / 32) words).
template <int MODE, bool WIDE>
__global__ __launch_bounds__(TR_THREADS, 3) void lftj_tri_wedge_kernel(const __grid_constant__ TriArgs A) {
    constexpr bool WRITE = MODE == 1;
    constexpr bool MATRIX = MODE == 2;
    extern __shared__ __align__(16) unsigned char tr_smem[];
    const int lane = threadIdx.x & 31;
    TrWarp<WIDE> &W = ((TrWarp<WIDE> *)tr_smem)[threadIdx.x >> 5];
    const uint32_t base = A.rank_base, nbits = A.rank_bits;
    const int32_t *d1 = A.T.data1;
    const int4 *dq = reinterpret_cast<const int4 *>(d1);
    for (uint32_t k = lane; k < TR_BITS / 32; k += 32) W.bm[k] = 0u;
    __syncwarp();
    unsigned long long cnt = 0, chk = 0;
    uint32_t qh = 0, qn = 0;   // queue head and length
    int32_t elo = 0, ehi = 0;  // ids of this lane's edge (a, b) in increasing order
    uint64_t eh = 0;           // hash prefix of elo
    uint64_t rowbase = 0;      // matrix mode: first word of this edge's row
    uint32_t ta32 = 0;         // matrix mode: start of T(a) in level 1
    // the first n queued hits, one per lane: the triangle (c, lo, hi) in
    // increasing id order (x, y, z), hashed from the prefix of x
    auto flush = [&](uint32_t n) {
        __syncwarp();
        const bool mine = (uint32_t)lane < n;
        int32_t c = 0;
        int src = 0;
        if (mine) tr_qget<WIDE>(W, qh + lane, c, src);
        const int32_t lo = __shfl_sync(AMJ_FULL_MASK, elo, src);
        const int32_t hi = __shfl_sync(AMJ_FULL_MASK, ehi, src);
        const uint64_t hlo = __shfl_sync(AMJ_FULL_MASK, eh, src);
        __syncwarp();
        if (mine) {
            const RankId r = A.hid[c];
            const bool first = r.id < lo;
            const int32_t x = first ? r.id : lo;
            const int32_t y = first ? lo : min(r.id, hi);
            const int32_t z = max(r.id, hi);
            cnt++;
            chk += amj_hash_step(amj_hash_step(first ? r.h1 : hlo, y), z);
            if (WRITE) {
                const unsigned m = __activemask();
                unsigned long long at = 0;
                if (lane == 0) at = atomicAdd(A.out_cursor, (unsigned long long)n);
                at = __shfl_sync(m, at, 0);
                if (at + lane < A.out_cap) {
                    A.out[0][at + lane] = x;
                    A.out[1][at + lane] = y;
                    A.out[2][at + lane] = z;
                }
            }
        }
        qh = (qh + n) & (TR_QCAP - 1);
        qn -= n;
    };
    // the current b: its children S(b) = sl_[0, db) have their bits set
    bool have_b = false;
    int32_t cur_b = 0;
    uint64_t db = 0;
    const int32_t *bl = nullptr;
    uint32_t nl = 0;   // children of b below the bitmap (a sorted prefix)
    auto set_bits = [&](int32_t b) {
        uint64_t sb, se;
        child_range(A.S, b, sb, se);
        db = se - sb;
        bl = d1 + sb;
        nl = 0;
        for (uint64_t k0 = 0; k0 < db; k0 += 128) {
            int32_t v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint64_t k = k0 + u * 32 + lane;
                v[u] = k < db ? bl[k] : 0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint64_t k = k0 + u * 32 + lane;
                const bool in = k < db;
                const uint32_t r = (uint32_t)v[u] - base;
                if (in && r < nbits) atomicOr(&W.bm[r >> 5], 1u << (r & 31));
                else if (in && k < TR_LOWCAP) W.low[k] = v[u];
                nl += __popc(__ballot_sync(AMJ_FULL_MASK, in && r >= nbits));
            }
        }
        __syncwarp();
    };
    auto clear_bits = [&]() {
        __syncwarp();
        for (uint64_t k0 = 0; k0 < db; k0 += 128) {
            int32_t v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint64_t k = k0 + u * 32 + lane;
                v[u] = k < db ? bl[k] : (int32_t)(base - 1);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint32_t r = (uint32_t)v[u] - base;
                if (r < nbits) W.bm[r >> 5] = 0u;
            }
        }
        __syncwarp();
    };
    while (true) {
        unsigned long long at = 0;
        if (lane == 0) at = atomicAdd(A.cursor_r, 32ull);
        at = __shfl_sync(AMJ_FULL_MASK, at, 0);
        if (at >= A.r_n) break;
        const uint64_t j = at + lane;
        const bool valid = j < A.r_n;
        int32_t b = 0;
        uint64_t ts = 0, te = 0;   // suffix of T(a) after b
        if (valid) {
            const uint64_t w = A.wedge[j];
            const uint32_t idx = (uint32_t)w;
            b = (int32_t)(w >> 32);
            const int32_t a = A.src1[idx];
            uint64_t ta;
            child_range(A.T, a, ta, te);
            ts = (uint64_t)idx + 1;
            if (MATRIX) {
                rowbase = A.moff[a] + ((uint64_t)idx - ta) * ((te - ta + 31) / 32);
                ta32 = (uint32_t)ta;
            } else {
                const RankId ra = A.hid[a], rb = A.hid[b];
                const bool alo = ra.id < rb.id;
                elo = alo ? ra.id : rb.id;
                ehi = alo ? rb.id : ra.id;
                eh = alo ? ra.h1 : rb.h1;
            }
        }
        // tl: first value of the suffix in the bitmap's ranks (the values
        // below form a short sorted prefix: gallop, then bisect)
        uint64_t tl = ts;
        if (te > ts && d1[ts] < (int32_t)base) {
            uint64_t lo = ts + 1, hi = te, step = 1;
            while (lo + step < te && d1[lo + step - 1] < (int32_t)base) {
                lo += step;
                step <<= 1;
            }
            if (lo + step < hi) hi = lo + step;
            while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if (d1[mid] < (int32_t)base) lo = mid + 1;
                else hi = mid;
            }
            tl = lo;
        }
        // quads of this edge's suffix part in the bitmap's ranks
        const uint32_t nq = te > tl ? (uint32_t)(((te + 3) >> 2) - (tl >> 2)) : 0u;
        const uint32_t qs = (uint32_t)(tl >> 2), h = (uint32_t)(tl & 3), len = (uint32_t)(te - tl);
        unsigned todo = __ballot_sync(AMJ_FULL_MASK, valid && te > ts);
        // the edges of one b form a run of lanes (the edges are sorted by b)
        while (todo) {
            const int32_t wb = __shfl_sync(AMJ_FULL_MASK, b, __ffs(todo) - 1);
            const unsigned run = todo & __ballot_sync(AMJ_FULL_MASK, b == wb);
            todo &= ~run;
            if (!have_b || wb != cur_b) {
                if (have_b) clear_bits();
                set_bits(wb);
                cur_b = wb;
                have_b = true;
            }
            if (db == 0) continue;
            const bool in_run = (run >> lane) & 1u;
            // suffix values below the bitmap (rare): binary search in S(b)'s low prefix
            const bool low_smem = nl <= TR_LOWCAP;
            unsigned lows = run & __ballot_sync(AMJ_FULL_MASK, tl > ts);
            while (lows) {
                const int l = __ffs(lows) - 1;
                lows &= lows - 1;
                const uint64_t wts = __shfl_sync(AMJ_FULL_MASK, ts, l);
                const uint64_t wtl = __shfl_sync(AMJ_FULL_MASK, tl, l);
                const uint64_t lrb = __shfl_sync(AMJ_FULL_MASK, rowbase, l);
                const uint32_t lta = __shfl_sync(AMJ_FULL_MASK, ta32, l);
                for (uint64_t k0 = wts; k0 < wtl; k0 += 32) {
                    const uint64_t k = k0 + lane;
                    bool hit = false;
                    int32_t c = 0;
                    if (k < wtl) {
                        c = d1[k];
                        hit = nl && (low_smem ? tr_sorted_find(W.low, nl, c) : tr_sorted_find(bl, nl, c));
                    }
                    if (MATRIX) {
                        if (hit) {
                            const uint32_t col = (uint32_t)k - lta;
                            atomicOr(&A.mtx[lrb + (col >> 5)], 1u << (col & 31));
                        }
                        continue;
                    }
                    const unsigned m = __ballot_sync(AMJ_FULL_MASK, hit);
                    if (hit) tr_qput<WIDE>(W, qh + qn + __popc(m & lanemask_lt()), c, l);
                    qn += __popc(m);
                    while (qn >= 32) flush(32);
                }
            }
            // the run's suffixes as one stream of quads: P = this edge's first
            // quad in the stream, Q = the stream's length
            const uint32_t x = in_run ? nq : 0u;
            const uint32_t incl = warp_inclusive_scan(x, lane);
            const uint32_t P = incl - x;
            const uint32_t Q = __shfl_sync(AMJ_FULL_MASK, incl, 31);
            const bool has = x > 0;
            const uint32_t qsh = qs | (h << 30);   // first quad (< 2^30) and head offset
            const uint32_t hl = h + len;           // suffix end, from the first quad's start
            const uint32_t pend = P + x;           // end of this edge's quads in the stream
            const unsigned hm = __ballot_sync(AMJ_FULL_MASK, has);
            for (uint32_t f0 = 0; f0 < Q; f0 += 32 * TR_UNROLL) {
                // this lane's quads f0 + TR_UNROLL * lane + t; the owner of the
                // first is the last lane whose quads start at or before it (the
                // starts P never decrease over the lanes)
                const uint32_t fl = f0 + TR_UNROLL * lane;
                int o = 0;
#pragma unroll
                for (int sft = 16; sft >= 1; sft >>= 1)
                    if (__shfl_sync(AMJ_FULL_MASK, P, o + sft) <= fl) o += sft;
                int4 cv[TR_UNROLL];
                uint32_t m4[TR_UNROLL], qi[TR_UNROLL];
                int own[TR_UNROLL];
                uint32_t oqsh = 0, oP = 0, ohl = 0, oe = 0;
#pragma unroll
                for (int u = 0; u < TR_UNROLL; u++) {
                    const uint32_t f = fl + u;
                    // quads of consecutive f cross at most one edge boundary
                    if (u > 0 && f >= oe) {
                        const unsigned rest = hm & ~(0xFFFFFFFFu >> (31 - o));
                        if (rest) o = __ffs(rest) - 1;
                    }
                    oqsh = __shfl_sync(AMJ_FULL_MASK, qsh, o);
                    oP = __shfl_sync(AMJ_FULL_MASK, P, o);
                    ohl = __shfl_sync(AMJ_FULL_MASK, hl, o);
                    oe = __shfl_sync(AMJ_FULL_MASK, pend, o);
                    own[u] = o;
                    const bool vq = f < Q;
                    const uint32_t rel = f - oP;
                    // values t of this quad inside the suffix: lo <= t < hi
                    const uint32_t e0 = 4 * rel;
                    const uint32_t lo = e0 == 0 ? (oqsh >> 30) : 0u;
                    const uint32_t hi = ohl > e0 ? (ohl - e0 < 4 ? ohl - e0 : 4u) : 0u;
                    m4[u] = vq && hi > lo ? ((0xFu >> (4 - hi)) & (0xFu << lo)) : 0u;
                    qi[u] = (oqsh & 0x3FFFFFFFu) + (vq ? rel : 0u);
                    cv[u] = dq[qi[u]];
                }
                uint32_t bits = 0;
#pragma unroll
                for (int u = 0; u < TR_UNROLL; u++) {
                    const uint32_t t4 = tr_bit(W.bm, cv[u].x, base) | (tr_bit(W.bm, cv[u].y, base) << 1) |
                                        (tr_bit(W.bm, cv[u].z, base) << 2) | (tr_bit(W.bm, cv[u].w, base) << 3);
                    bits |= (t4 & m4[u]) << (4 * u);
                }
                if (MATRIX) {
                    // value t of quad qi sits at level-1 position 4 qi + t
#pragma unroll
                    for (int u = 0; u < TR_UNROLL; u++) {
                        const uint64_t orb = __shfl_sync(AMJ_FULL_MASK, rowbase, own[u]);
                        const uint32_t ota = __shfl_sync(AMJ_FULL_MASK, ta32, own[u]);
#pragma unroll
                        for (int t = 0; t < 4; t++)
                            if ((bits >> (4 * u + t)) & 1u) {
                                const uint32_t col = 4 * qi[u] + t - ota;
                                atomicOr(&A.mtx[orb + (col >> 5)], 1u << (col & 31));
                            }
                    }
                    continue;
                }
                const uint32_t nh = __popc(bits);
                const uint32_t hincl = warp_inclusive_scan(nh, lane);
                const uint32_t tot = __shfl_sync(AMJ_FULL_MASK, hincl, 31);
                if (tot) {
                    if (qn + tot > TR_QCAP) flush(qn);   // (nearly every value a hit) make room
                    uint32_t pos = qh + qn + hincl - nh;
#pragma unroll
                    for (int u = 0; u < TR_UNROLL; u++) {
                        if ((bits >> (4 * u)) & 1u) tr_qput<WIDE>(W, pos++, cv[u].x, own[u]);
                        if ((bits >> (4 * u + 1)) & 1u) tr_qput<WIDE>(W, pos++, cv[u].y, own[u]);
                        if ((bits >> (4 * u + 2)) & 1u) tr_qput<WIDE>(W, pos++, cv[u].z, own[u]);
                        if ((bits >> (4 * u + 3)) & 1u) tr_qput<WIDE>(W, pos++, cv[u].w, own[u]);
                    }
                    qn += tot;
                    while (qn >= 32) flush(32);
                }
            }
        }
        if (qn) flush(qn);
    }
    if (have_b) clear_bits();
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if (lane == 0 && cnt) {
        atomicAdd(A.count, cnt);
        atomicAdd(A.checksum, chk);
    }
}

// words of every vertex a's matrix (d+(a) rows of ceil(d+(a) / 32) words),
// indexed by a's rank; the scan turns them into first words
__global__ void matrix_words_kernel(const int32_t *__restrict__ data0, const uint64_t *__restrict__ off0,
                                    uint64_t len0, uint64_t *__restrict__ words) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len0; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = off0[i + 1] - off0[i];
        words[(uint32_t)data0[i]] = k * ((k + 31) / 32);
    }
}

// The triangle matrices of a degree-ranked trie R (ranks 0..nv-1): row x of
// vertex a's matrix has bit y for every triangle (a, x, y), x and y counted
// from the start of T(a).  *moff gets the first word of each matrix; the
// matrices need *words 32-bit words.  Fails with AMJ_ENOMEM beyond max_words.
int lftj_tri_matrices(amj_ctx *ctx, const Trie2 &R, const uint64_t *wedge, uint64_t nv, uint32_t rank_bits,
                      uint64_t max_words, DBuf<uint64_t> *moff, uint32_t **mtx, uint64_t *words) {
    AMJ_TRY(moff->alloc(ctx, nv + 1));
    AMJ_CUDA_TRY(cudaMemsetAsync(moff->p, 0, (nv + 1) * sizeof(uint64_t), ctx->stream));
    if (R.len0) {
        note_launch(ctx);
        matrix_words_kernel<<<(unsigned)std::min<uint64_t>((R.len0 + 255) / 256, (uint64_t)ctx->num_sms * 16), 256,
                              0, ctx->stream>>>(R.data0.p, R.off0.p, R.len0, moff->p);
        AMJ_CUDA_TRY(cudaGetLastError());
    }
    AMJ_TRY(scan_exclusive_u64(ctx, moff->p, moff->p, nv + 1, nullptr));
    AMJ_CUDA_TRY(cudaMemcpyAsync(words, moff->p + nv, sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (*words > max_words) return fail(AMJ_ENOMEM, "LFTJ 4-clique: the triangle matrices do not fit");
    // the matrices live in one buffer the context keeps between calls (they
    // are the largest allocation of the query; allocating them anew every
    // call stalled the host while the device memory pool grew)
    const uint64_t need = *words ? *words : 1;
    if (ctx->c4_mtx_words < need) {
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (ctx->c4_mtx) (void)cudaFree(ctx->c4_mtx);
        ctx->c4_mtx = nullptr;
        ctx->c4_mtx_words = 0;
        if (cudaMalloc(&ctx->c4_mtx, need * sizeof(uint32_t)) != cudaSuccess) {
            (void)cudaGetLastError();
            ctx->c4_mtx = nullptr;
            return fail(AMJ_ENOMEM, "LFTJ 4-clique: the triangle matrices do not fit");
        }
        ctx->c4_mtx_words = need;
    }
    *mtx = static_cast<uint32_t *>(ctx->c4_mtx);
    AMJ_CUDA_TRY(cudaMemsetAsync(*mtx, 0, need * sizeof(uint32_t), ctx->stream));
    if (R.len1 == 0) return AMJ_OK;
    if (reinterpret_cast<uintptr_t>(R.data1.p) & 15) return fail(AMJ_ECUDA, "LFTJ: trie level 1 is not 16-byte aligned");
    DBuf<unsigned long long> cursor;
    AMJ_TRY(cursor.alloc(ctx, 1));
    AMJ_CUDA_TRY(cudaMemsetAsync(cursor.p, 0, sizeof(unsigned long long), ctx->stream));
    TriArgs A{};
    A.r_src = R.src1.p;
    A.r_dst = R.data1.p;
    A.r_n = R.len1;
    A.S = A.T = A.R = trie_ref(R);
    A.r_lo = 0;
    A.r_hi = R.len1;
    A.sorted_out = 1;
    A.wedge = wedge;
    A.src1 = R.src1.p;
    A.moff = moff->p;
    A.mtx = *mtx;
    A.cursor_r = cursor.p;
    uint32_t bits = TR_BITS;
    if (rank_bits && rank_bits < bits) bits = rank_bits < 32 ? 32u : rank_bits;
    if (nv < bits) bits = (uint32_t)((nv + 31) / 32 * 32);
    A.rank_bits = bits;
    A.rank_base = (uint32_t)(nv > bits ? nv - bits : 0);
    auto kr = lftj_tri_wedge_kernel<2, false>;
    constexpr size_t smem = tr_smem<false>();
    AMJ_CUDA_TRY(cudaFuncSetAttribute(kr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    AMJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kr, TR_THREADS, smem));
    if (per_sm < 1) per_sm = 1;
    note_launch(ctx);
    kr<<<(unsigned)(ctx->num_sms * per_sm), TR_THREADS, smem, ctx->stream>>>(A);
    AMJ_CUDA_TRY(cudaGetLastError());
    return AMJ_OK;
}

// (b << 32 | entry) for every level-1 entry (a, b) of R
__global__ void wedge_keys_kernel(const int32_t *__restrict__ data1, uint64_t n, uint64_t *__restrict__ keys) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        keys[i] = ((uint64_t)(uint32_t)data1[i] << 32) | i;
}

// The level-1 entries of a degree-ranked trie grouped by b: a stable sort
// of (b << 32 | entry) on the rank bits of b.
int build_wedges(amj_ctx *ctx, const Trie2 &R, uint64_t nv, DBuf<uint64_t> *out) {
    const uint64_t n = R.len1;
    if (n >= (1ull << 32)) return fail(AMJ_EUNSUPPORTED, "LFTJ: 2^32 or more edges");
    DBuf<uint64_t> other;
    AMJ_TRY(out->alloc(ctx, n ? n : 1));
    if (n == 0) return AMJ_OK;
    AMJ_TRY(other.alloc(ctx, n));
    note_launch(ctx);
    wedge_keys_kernel<<<(unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->num_sms * 16), 256, 0,
                        ctx->stream>>>(R.data1.p, n, out->p);
    AMJ_CUDA_TRY(cudaGetLastError());
    int bits = 1;
    while (bits < 32 && (nv - 1) >> bits) bits++;
    uint64_t *sorted = nullptr;
    AMJ_TRY(radix_sort_u64(ctx, out->p, other.p, n, SK_IDENT, 32, 32 + bits, &sorted));
    if (sorted != out->p) std::swap(*out, other);   // the sorted buffer becomes the result
    return AMJ_OK;
}

template <bool WRITE>
__global__ __launch_bounds__(256) void lftj_tri_dfs_kernel(const __grid_constant__ TriArgs A) {
    const int lane = threadIdx.x & 31;
    unsigned long long cnt = 0, chk = 0;
    while (true) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(A.cursor, 32ull);
        base = __shfl_sync(AMJ_FULL_MASK, base, 0);
        if (base >= A.r_n) break;
        const uint64_t j = base + lane;
        const bool valid = j < A.r_n;
        int32_t a = 0, b = 0;
        uint64_t sb = 0, eb = 0, ta = 0, ea = 0;
        if (valid) {
            a = A.r_src[j];
            b = A.r_dst[j];
            child_range(A.S, b, sb, eb);
            if (eb > sb) child_range(A.T, a, ta, ea);
            if (A.heavy_deg && ea > ta) {
                uint64_t rs, re;
                child_range(A.R, a, rs, re);
                int32_t lo;
                uint32_t span;
                if (heavy_vertex(A, re - rs, ta, ea, lo, span)) sb = eb = 0;  // the bitmap kernel owns this edge
            }
        }
        const uint64_t lb = eb - sb, la = ea - ta;
        const bool active = valid && lb && la;
        const bool small = active && (lb + la <= (uint64_t)A.small_sum);
        const uint64_t hab = amj_hash_step(amj_hash_step(AMJ_CHECKSUM_SEED, a), b);
        // lane-local merge of short pairs
        if (!WRITE) {
            if (small) {
                uint64_t p = sb, q = ta;
                while (p < eb && q < ea) {
                    const int32_t x = A.S.data1[p], y = A.T.data1[q];
                    if (x == y) {
                        cnt++;
                        chk += tri_chk(A, hab, a, b, x);
                        p++;
                        q++;
                    } else if (x < y) p++;
                    else q++;
                }
            }
        } else {
            // count, reserve once per warp, then write
            uint32_t mine = 0;
            if (small) {
                uint64_t p = sb, q = ta;
                while (p < eb && q < ea) {
                    const int32_t x = A.S.data1[p], y = A.T.data1[q];
                    if (x == y) { mine++; p++; q++; }
                    else if (x < y) p++;
                    else q++;
                }
            }
            const uint32_t incl = warp_inclusive_scan(mine, lane);
            const uint32_t tot = __shfl_sync(AMJ_FULL_MASK, incl, 31);
            unsigned long long wbase = 0;
            if (lane == 0 && tot) wbase = atomicAdd(A.out_cursor, (unsigned long long)tot);
            wbase = __shfl_sync(AMJ_FULL_MASK, wbase, 0);
            unsigned long long pos = wbase + incl - mine;
            if (small && mine) {
                uint64_t p = sb, q = ta;
                while (p < eb && q < ea) {
                    const int32_t x = A.S.data1[p], y = A.T.data1[q];
                    if (x == y) {
                        if (pos < A.out_cap) tri_store(A, pos, a, b, x);
                        pos++;
                        cnt++;
                        chk += tri_chk(A, hab, a, b, x);
                        p++; q++;
                    } else if (x < y) p++;
                    else q++;
                }
            }
        }
        // warp-cooperative intersection of long pairs
        unsigned big = __ballot_sync(AMJ_FULL_MASK, active && !small);
        while (big) {
            const int l = __ffs(big) - 1;
            big &= big - 1;
            const int32_t wa = __shfl_sync(AMJ_FULL_MASK, a, l);
            const int32_t wb = __shfl_sync(AMJ_FULL_MASK, b, l);
            const uint64_t wsb = __shfl_sync(AMJ_FULL_MASK, sb, l), web = __shfl_sync(AMJ_FULL_MASK, eb, l);
            const uint64_t wta = __shfl_sync(AMJ_FULL_MASK, ta, l), wea = __shfl_sync(AMJ_FULL_MASK, ea, l);
            const uint64_t whab = __shfl_sync(AMJ_FULL_MASK, hab, l);
            if (!WRITE) {
                warp_intersect(A.S.data1 + wsb, web - wsb, A.T.data1 + wta, wea - wta, lane, [&](int32_t c) {
                    cnt++;
                    chk += tri_chk(A, whab, wa, wb, c);
                });
            } else {
                // one reservation per round: count this round's matches with a ballot inside emit
                warp_intersect(A.S.data1 + wsb, web - wsb, A.T.data1 + wta, wea - wta, lane, [&](int32_t c) {
                    cnt++;
                    chk += tri_chk(A, whab, wa, wb, c);
                    const unsigned long long p = atomicAdd(A.out_cursor, 1ull);
                    if (p < A.out_cap) tri_store(A, p, wa, wb, c);
                });
            }
        }
    }
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if (lane == 0 && cnt) {
        atomicAdd(A.count, cnt);
        atomicAdd(A.checksum, chk);
    }
}

// ---- BFS ----

// candidates of entry j: the shorter child list of (S(b), T(a)); 0 when either is empty
// (wedge form: T(a)'s values after b, when S(b) is not empty)
__global__ void lftj_tri_bfs_count_kernel(const __grid_constant__ TriArgs A, unsigned long long *cand) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < A.r_n; j += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t sb, eb, ta = 0, ea = 0;
        child_range(A.S, A.r_dst[j], sb, eb);
        if (eb > sb) child_range(A.T, A.r_src[j], ta, ea);
        const uint64_t lb = eb - sb, la = ea - ta;
        if (A.bfs_wedge) {
            const uint64_t g = A.r_lo + j;   // the entry's position in T(a)
            cand[j] = (lb && ea > g + 1) ? ea - g - 1 : 0ull;
        } else {
            cand[j] = (lb && la) ? (lb < la ? lb : la) : 0ull;
        }
    }
}

constexpr int BFS_TILE = 2048;
constexpr int BFS_THREADS = 256;
constexpr int BFS_SMEM_ENTRIES = 2048;
constexpr int BFS_RUN = BFS_TILE / BFS_THREADS;   // consecutive candidates per thread

__device__ __forceinline__ uint64_t upper_bound_u64(const unsigned long long *a, uint64_t lo, uint64_t hi,
                                                    unsigned long long v) {
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (a[mid] <= v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

template <bool WRITE>
__global__ __launch_bounds__(BFS_THREADS) void lftj_tri_bfs_expand_kernel(const __grid_constant__ TriArgs A,
                                                                          const unsigned long long *__restrict__ offs,
                                                                          unsigned long long total) {
    __shared__ unsigned long long s_off[BFS_SMEM_ENTRIES + 1];
    __shared__ uint64_t s_e0, s_e1;
    unsigned long long cnt = 0, chk = 0;
    const int lane = threadIdx.x & 31;
    for (unsigned long long tile = blockIdx.x * (unsigned long long)BFS_TILE; tile < total;
         tile += (unsigned long long)gridDim.x * BFS_TILE) {
        const unsigned long long tend = (tile + BFS_TILE < total) ? tile + BFS_TILE : total;
        if (threadIdx.x == 0) {
            // entries owning candidates tile .. tend-1: offs[e] <= t < offs[e+1]
            s_e0 = upper_bound_u64(offs, 0, A.r_n, tile) - 1;
            s_e1 = upper_bound_u64(offs, 0, A.r_n, tend - 1) - 1;
        }
        __syncthreads();
        const uint64_t e0 = s_e0, e1 = s_e1;
        const uint64_t ne = e1 - e0 + 1;
        const bool in_smem = ne <= BFS_SMEM_ENTRIES;
        if (in_smem)
            for (uint64_t k = threadIdx.x; k < ne; k += BFS_THREADS) s_off[k] = offs[e0 + k];
        __syncthreads();
        // each thread takes a run of BFS_RUN consecutive candidates: its
        // edge is searched once, then followed forward, and the edge's child
        // ranges and ids are read when the edge changes
        const unsigned long long t0 = tile + (unsigned long long)threadIdx.x * BFS_RUN;
        const unsigned long long t1 = t0 + BFS_RUN < tend ? t0 + BFS_RUN : tend;
        uint64_t e = ~0ull, sb = 0, eb = 0, ta = 0, ea = 0, nxt = 0, cur = 0;
        int32_t a = 0, b = 0, xa = 0, xb = 0;
        uint64_t hab = 0;
        bool s_short = false;
        for (unsigned long long t = t0; t < t1; t++) {
            if (e == ~0ull || t >= nxt) {
                if (e == ~0ull) {
                    if (in_smem) {
                        uint64_t lo = 0, hi = ne;
                        while (lo < hi) {
                            uint64_t mid = (lo + hi) >> 1;
                            if (s_off[mid] <= t) lo = mid + 1;
                            else hi = mid;
                        }
                        e = e0 + lo - 1;
                    } else {
                        e = upper_bound_u64(offs, e0, e1 + 1, t) - 1;
                    }
                } else {
                    do e++;
                    while (offs[e + 1] <= t);   // edges without candidates are passed over
                }
                cur = offs[e];
                nxt = offs[e + 1];
                a = A.r_src[e];
                b = A.r_dst[e];
                child_range(A.S, b, sb, eb);
                child_range(A.T, a, ta, ea);
                // expand the shorter list, search the longer (wedge form:
                // expand T(a) after b, search S(b))
                s_short = !A.bfs_wedge && (eb - sb) <= (ea - ta);
                xa = A.inv ? A.inv[a] : a;
                xb = A.inv ? A.inv[b] : b;
                hab = amj_hash_step(amj_hash_step(AMJ_CHECKSUM_SEED, xa), xb);
            }
            const unsigned long long k = t - cur;
            const int32_t c = s_short ? A.S.data1[sb + k]
                                      : A.T.data1[(A.bfs_wedge ? A.r_lo + e + 1 : ta) + k];
            const int32_t *hay = s_short ? A.T.data1 : A.S.data1;
            uint64_t lo = s_short ? ta : sb, hi = s_short ? ea : eb;
            while (lo < hi) {
                uint64_t mid = (lo + hi) >> 1;
                if (hay[mid] < c) lo = mid + 1;
                else hi = mid;
            }
            const bool found = lo < (s_short ? ea : eb) && hay[lo] == c;
            if (found) {
                const int32_t xc = A.inv ? A.inv[c] : c;
                cnt++;
                chk += tri_chk(A, hab, xa, xb, xc);
                if (WRITE) {
                    const unsigned long long p = atomicAdd(A.out_cursor, 1ull);
                    if (p < A.out_cap) tri_store(A, p, xa, xb, xc);
                }
            }
        }
        __syncthreads();
    }
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if (lane == 0 && cnt) {
        atomicAdd(A.count, cnt);
        atomicAdd(A.checksum, chk);
    }
}

// ---- host side ----

struct LftjCounters {
    unsigned long long cursor, count, checksum, out_cursor, cursor0, cursor_r, heavy_n;
};


// Run the triangle join over tries R, S, T (R's level-1 entries are the
// (a,b) pairs).  Count + checksum always; with `out` non-null the tuples are
// written too (out_cap rows available).
int lftj_triangle(amj_ctx *ctx, const Trie2 &R, const Trie2 &S, const Trie2 &T, int algo, int32_t *const *out,
                  uint64_t out_cap, uint64_t *count, uint64_t *checksum, uint64_t *written, int small_sum,
                  uint64_t r_lo, uint64_t r_hi, uint32_t heavy_deg, double *kernel_ms, int sorted_out,
                  const int32_t *inv, const uint64_t *wedge, uint64_t nv, uint32_t rank_bits) {
    bool timed[2] = {false, false};
    TriArgs A{};
    A.sorted_out = sorted_out;
    if (r_hi > R.len1) r_hi = R.len1;
    if (r_lo > r_hi) r_lo = r_hi;
    A.r_src = R.src1.p + r_lo;
    A.r_dst = R.data1.p + r_lo;
    A.r_n = r_hi - r_lo;
    A.S = trie_ref(S);
    A.T = trie_ref(T);
    A.R = trie_ref(R);
    A.r_lo = r_lo;
    A.r_hi = r_hi;
    A.small_sum = small_sum;
    DBuf<LftjCounters> ctr;
    AMJ_TRY(ctr.alloc(ctx, 1));
    AMJ_CUDA_TRY(cudaMemsetAsync(ctr.p, 0, sizeof(LftjCounters), ctx->stream));
    A.cursor = &ctr.p->cursor;
    A.count = &ctr.p->count;
    A.checksum = &ctr.p->checksum;
    A.out_cursor = &ctr.p->out_cursor;
    A.cursor0 = &ctr.p->cursor0;
    DBuf<uint32_t> heavy;
    DBuf<RankId> hid;
    A.cursor_r = &ctr.p->cursor_r;
    const bool write = out != nullptr;
    if (write) {
        for (int i = 0; i < 3; i++) A.out[i] = out[i];
        A.out_cap = out_cap;
    }
    if (A.r_n) {
        if (algo == AMJ_LFTJ_DFS) {
            // a degree-ranked trie goes to the wedge kernel alone
            const bool rest = inv == nullptr;
            AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[0], ctx->stream));
            if (inv) {
                if (reinterpret_cast<uintptr_t>(S.data1.p) & 15)
                    return fail(AMJ_ECUDA, "LFTJ: trie level 1 is not 16-byte aligned");
                uint32_t bits = TR_BITS;
                if (rank_bits && rank_bits < bits) bits = rank_bits < 32 ? 32u : rank_bits;
                if (nv < bits) bits = (uint32_t)((nv + 31) / 32 * 32);
                if (bits == 0) bits = 32;
                A.inv = inv;
                A.wedge = wedge + r_lo;
                A.src1 = R.src1.p;
                A.rank_bits = bits;
                A.rank_base = (uint32_t)(nv > bits ? nv - bits : 0);
                AMJ_TRY(hid.alloc(ctx, nv));
                note_launch(ctx);
                rank_ids_kernel<<<(unsigned)std::min<uint64_t>((nv + 255) / 256, (uint64_t)ctx->num_sms * 16), 256,
                                  0, ctx->stream>>>(inv, nv, hid.p);
                AMJ_CUDA_TRY(cudaGetLastError());
                A.hid = hid.p;
                const bool wide = nv > TR_NARROW_RANKS;
                auto kr = wide ? (write ? lftj_tri_wedge_kernel<1, true> : lftj_tri_wedge_kernel<0, true>)
                               : (write ? lftj_tri_wedge_kernel<1, false> : lftj_tri_wedge_kernel<0, false>);
                const size_t smem = wide ? tr_smem<true>() : tr_smem<false>();
                AMJ_CUDA_TRY(cudaFuncSetAttribute(kr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                int per_sm = 0;
                AMJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kr, TR_THREADS, smem));
                if (per_sm < 1) per_sm = 1;
                note_launch(ctx);
                kr<<<(unsigned)(ctx->num_sms * per_sm), TR_THREADS, smem, ctx->stream>>>(A);
                AMJ_CUDA_TRY(cudaGetLastError());
                timed[0] = true;
            }
            if (rest && heavy_deg) {
                // the bitmap kernel takes the heavy vertices; its shared memory: bitmap + 1024 x 24 B
                const uint32_t bits_max = 1u << 20;
                const size_t smem = (size_t)bits_max / 8 + (size_t)BM_THREADS * (8 + 8 + 4 + 4 + 4);
                if (smem <= (size_t)ctx->max_smem_optin && R.len0) {
                    A.heavy_deg = heavy_deg;
                    A.bitmap_bits = bits_max;
                    AMJ_TRY(heavy.alloc(ctx, R.len0));
                    A.heavy_list = heavy.p;
                    A.heavy_n = &ctr.p->heavy_n;
                    note_launch(ctx);
                    heavy_list_kernel<<<(unsigned)std::min<uint64_t>((R.len0 + 255) / 256, (uint64_t)ctx->num_sms * 8), 256, 0,
                                        ctx->stream>>>(A, heavy.p, &ctr.p->heavy_n);
                    AMJ_CUDA_TRY(cudaGetLastError());
                    auto kb = write ? lftj_tri_bitmap_kernel<true> : lftj_tri_bitmap_kernel<false>;
                    AMJ_CUDA_TRY(cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                    note_launch(ctx);
                    kb<<<(unsigned)ctx->num_sms, BM_THREADS, smem, ctx->stream>>>(A);
                    AMJ_CUDA_TRY(cudaGetLastError());
                    timed[0] = true;
                }
            }
            AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[1], ctx->stream));
            if (rest) {
                int per_sm = 0;
                AMJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &per_sm, write ? lftj_tri_dfs_kernel<true> : lftj_tri_dfs_kernel<false>, 256, 0));
                if (per_sm < 1) per_sm = 1;
                const unsigned grid = (unsigned)(ctx->num_sms * per_sm);
                note_launch(ctx);
                AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[2], ctx->stream));
                if (write) lftj_tri_dfs_kernel<true><<<grid, 256, 0, ctx->stream>>>(A);
                else lftj_tri_dfs_kernel<false><<<grid, 256, 0, ctx->stream>>>(A);
                AMJ_CUDA_TRY(cudaGetLastError());
                AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[3], ctx->stream));
                timed[1] = true;
            }
        } else {
            // a degree-ranked trie (ranks as vertex ids): wedge candidates, ids mapped back
            A.bfs_wedge = inv != nullptr && &R == &S && &S == &T;
            A.inv = inv;
            DBuf<unsigned long long> cand;
            AMJ_TRY(cand.alloc(ctx, A.r_n + 1));
            const unsigned g1 = (unsigned)std::min<uint64_t>((A.r_n + 255) / 256, (uint64_t)ctx->num_sms * 16);
            note_launch(ctx);
            AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[0], ctx->stream));
            lftj_tri_bfs_count_kernel<<<g1, 256, 0, ctx->stream>>>(A, cand.p);
            AMJ_CUDA_TRY(cudaGetLastError());
            AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[1], ctx->stream));
            timed[0] = true;
            AMJ_TRY(scan_exclusive_u64(ctx, (const uint64_t *)cand.p, (uint64_t *)cand.p, A.r_n,
                                       (uint64_t *)cand.p + A.r_n));
            unsigned long long total = 0;
            AMJ_CUDA_TRY(cudaMemcpyAsync(&total, cand.p + A.r_n, sizeof(total), cudaMemcpyDeviceToHost, ctx->stream));
            AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
            if (total) {
                int per_sm = 0;
                AMJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &per_sm, write ? lftj_tri_bfs_expand_kernel<true> : lftj_tri_bfs_expand_kernel<false>,
                    BFS_THREADS, 0));
                if (per_sm < 1) per_sm = 1;
                const uint64_t tiles = (total + BFS_TILE - 1) / BFS_TILE;
                const unsigned grid = (unsigned)std::min<uint64_t>(tiles, (uint64_t)ctx->num_sms * per_sm);
                note_launch(ctx);
                AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[2], ctx->stream));
                if (write)
                    lftj_tri_bfs_expand_kernel<true><<<grid, BFS_THREADS, 0, ctx->stream>>>(A, cand.p, total);
                else
                    lftj_tri_bfs_expand_kernel<false><<<grid, BFS_THREADS, 0, ctx->stream>>>(A, cand.p, total);
                AMJ_CUDA_TRY(cudaGetLastError());
                AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[3], ctx->stream));
                timed[1] = true;
            }
        }
    }
    LftjCounters h{};
    AMJ_CUDA_TRY(cudaMemcpyAsync(&h, ctr.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    *count = h.count;
    *checksum = h.checksum;
    if (written) *written = write ? (h.out_cursor < out_cap ? h.out_cursor : out_cap) : 0;
    if (kernel_ms) {
        if (timed[0]) kernel_ms[0] += event_ms(ctx->kev[0], ctx->kev[1]);
        if (timed[1]) kernel_ms[1] += event_ms(ctx->kev[2], ctx->kev[3]);
    }
    return AMJ_OK;
}

}  // namespace amj
