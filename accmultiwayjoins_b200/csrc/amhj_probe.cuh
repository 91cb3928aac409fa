// AMHJ multi-way probe: device-side plan, frontier layout and the probe
// kernel template.  Included by amhj.cu only.
//
// Reference: AMHJ_count / AMHJ_write (MHJ-GPU/Joins/AMHJ.cuh:20-280) run one
// warp per probe tuple and a depth-first search with backtracking over the
// build tables; at each level the warp scans a bucket 32 slots at a time and
// keeps up to 32 matches (common_kernels.cuh:27-67).
//
// Here a warp runs the depth-first search over *frontiers* of up to 32
// partial tuples: depth 0 holds 32 probe tuples, depth d+1 the matches of one
// 32-candidate chunk of depth d.  The candidates of a frontier are the
// concatenation of its entries' bucket ranges; every lane takes one candidate
// (owner found by a 5-step binary search over the entries' prefix sums in
// shared memory), so all 32 lanes work even when buckets hold 1-4 rows, and
// the rows of a bucket are read by consecutive lanes (coalesced).  Matches are
// compacted with a ballot into the next frontier, whose bucket ranges the
// matching lanes look up in parallel.  At the last depth matches are counted
// (with the tuple checksum) or written with one output reservation per warp
// per chunk.  Work sharing splits candidate ranges longer than twice the task
// size: the entry keeps one task's worth and the rest goes to a device task
// queue as two halves; idle warps pop tasks.  Every wait in the kernel is
// bounded by %globaltimer and reports into the status block.
#pragma once
#include "amj_ops.cuh"

namespace amj {

constexpr int PROBE_THREADS = 256;
constexpr int PROBE_WARPS = PROBE_THREADS / 32;

struct LevelDesc {
    const uint32_t *buc_ptrs;
    const int32_t *col[4];
    const int2 *slots;
    uint32_t mask;
    int8_t layout, key_mode, ncols, npad;
    int8_t key_attr[2];
    uint8_t cmp_mask, bind_mask;
    int8_t attr[4];
};

struct alignas(16) ProbePlan {
    uint64_t row_lo, row_hi;            // probe rows handled by this launch
    const int32_t *probe_col[AMJ_MAX_COLS];
    int8_t probe_attr[AMJ_MAX_COLS];
    int8_t probe_ncols, L, k, pad0;
    LevelDesc lv[AMJ_MAX_BUILD_TABLES];
    // Inline filters: a level that binds nothing and is looked up by the
    // pair of its columns (C(0,2) of the triangle, D/E/F of the 4-clique) is
    // evaluated by the lane that created the partial tuple instead of
    // becoming a frontier depth; its number of exact matches multiplies the
    // tuple's weight.  next_lv[d] / prev_lv[d]: the next / previous level
    // that is a frontier depth (L / -1 at the ends).
    uint8_t inl[AMJ_MAX_BUILD_TABLES];
    int8_t next_lv[AMJ_MAX_BUILD_TABLES];
    int8_t prev_lv[AMJ_MAX_BUILD_TABLES];
    uint8_t has_inl;                    // any level inlined: run the weighted kernels
    uint8_t sort_out;                   // TRI / FOUR over the degree-ordered copy of an oriented
                                        // relation: every tuple is reported with its values sorted
    // bind_col[d][a]: the column of level d that binds attribute a, or -1
    // (the value then comes from the frontier)
    int8_t bind_col[AMJ_MAX_BUILD_TABLES][AMJ_MAX_ATTRS];
    int32_t *out[AMJ_MAX_ATTRS];
    uint64_t out_cap;
    uint32_t task_chunk;
    uint32_t task_cap;
    uint64_t spin_limit_ns;
    uint32_t depth_bytes;               // shared memory per frontier
    uint32_t warp_bytes;                // shared memory per warp
    // DRO: units that overflowed the output are recorded for the residual pass
    uint32_t dro;                       // 1: main pass of direct result output
    uint32_t unit_cap;
    // work sharing at level 0: the level-0 candidates of rows row_lo..row_hi-1
    // form one space (l0_start[r - row_lo] = first candidate of row r,
    // l0_start[rows] = total); units are 32-candidate chunks of it
    const unsigned long long *l0_start;
    uint32_t lbs;
    // frequent-item buffering: a depth-fib_level entry whose key is one of
    // the cached frequent keys takes its suffix tuples from the cache
    const int32_t *fib_keys;               // hash set of frequent keys, fib_mask+1 slots
    const uint32_t *fib_slot_idx;          // cache index of the key in each slot
    const unsigned long long *fib_off;     // suffix tuples of key i: [fib_off[i], fib_off[i+1])
    const int32_t *fib_cols[AMJ_MAX_ATTRS];
    uint32_t fib_mask;
    uint32_t fib_suffix_attrs;             // attributes the cached tuples provide
    int32_t fib_level;                     // -1: off
};
static_assert(sizeof(ProbePlan) % 16 == 0, "plans are copied as 16-byte words");

struct ProbeState {
    unsigned long long next_batch;
    unsigned long long count;
    unsigned long long checksum;
    unsigned long long out_cursor;
    unsigned long long overflow_rows;
    unsigned int q_head, q_tail;
    unsigned int busy;
    unsigned int n_units;
    unsigned long long tasks_pushed, tasks_popped;
    unsigned long long fib_rows;
};

struct Task {
    int32_t vals[AMJ_MAX_ATTRS];
    uint32_t s, aux, sz;
    uint32_t w;         // weight (multiplicity) of the entry
    uint8_t depth, m8;
    uint16_t qid;       // query of a batched launch (0 for a single query)
};

// DRO breakpoint: a unit (probe batch or task) whose output did not fit; the
// residual pass re-enumerates it, skipping the `written` rows it already wrote.
struct Breakpoint {
    uint32_t kind;      // 0 probe batch, 1 task, 2 level-0 chunk
    uint32_t id;        // batch number, task slot or chunk number
    unsigned long long written;
};

// ---- shared-memory frontier of one depth ----
// vals[k][32] int32 | s[32] u32 | aux[32] u32 | w[32] u32 | psum[32] u64 | meta | m8[32] u8
struct Frontier {
    int32_t *vals;
    uint32_t *s;
    uint32_t *aux;
    uint32_t *w;                // weight: how many identical tuples the entry stands for
    unsigned long long *psum;
    uint8_t *m8;
    unsigned long long *meta;   // [0] cursor, [1] total, [2] n
};

__device__ __forceinline__ Frontier frontier_at(char *wbase, const ProbePlan &P, int d) {
    char *p = wbase + (uint32_t)d * P.depth_bytes;
    Frontier f;
    f.vals = (int32_t *)p;
    p += 128 * P.k;
    f.s = (uint32_t *)p;
    p += 128;
    f.aux = (uint32_t *)p;
    p += 128;
    f.w = (uint32_t *)p;
    p += 128;
    f.psum = (unsigned long long *)p;
    p += 256;
    f.meta = (unsigned long long *)p;
    p += 32;
    f.m8 = (uint8_t *)p;
    return f;
}

constexpr uint8_t FIB_FLAG = 0x80;   // frontier entry served from the frequent-item cache

// sort the tuple of a TRI (k = 3) or FOUR (k = 4) query: a sorting network
__device__ __forceinline__ void sort_tuple(int32_t *tv, int k) {
    auto cs = [&](int i, int j) {
        if (tv[i] > tv[j]) {
            const int32_t t = tv[i];
            tv[i] = tv[j];
            tv[j] = t;
        }
    };
    if (k == 3) {
        cs(0, 1);
        cs(1, 2);
        cs(0, 1);
    } else if (k == 4) {
        cs(0, 1);
        cs(2, 3);
        cs(0, 2);
        cs(1, 3);
        cs(1, 2);
    }
}

// cache index of a frequent key, or -1
__device__ __forceinline__ int fib_find(const ProbePlan &P, int32_t key) {
    uint32_t s = hash_key(key) & P.fib_mask;
    for (uint32_t n = 0; n <= P.fib_mask; n++) {
        const int32_t k = P.fib_keys[s];
        if (k == key) return (int)P.fib_slot_idx[s];
        if (k == OA_EMPTY_KEY) return -1;
        s = (s + 1) & P.fib_mask;
    }
    return -1;
}

__host__ __device__ inline uint32_t frontier_bytes(int k) { return 128u * k + 128 + 128 + 128 + 256 + 32 + 32; }

// Fill inl / next_lv / prev_lv of a plan whose levels are set.  Level 0 is
// never inlined (the probe rows create its entries).
__host__ inline void plan_inline(ProbePlan &P) {
    for (int l = 0; l < AMJ_MAX_BUILD_TABLES; l++) {
        P.inl[l] = 0;
        P.next_lv[l] = (int8_t)P.L;
        P.prev_lv[l] = -1;
    }
    for (int l = 0; l < AMJ_MAX_BUILD_TABLES; l++)
        for (int a = 0; a < AMJ_MAX_ATTRS; a++) P.bind_col[l][a] = -1;
    for (int l = 0; l < P.L; l++)
        for (int c = 0; c < P.lv[l].ncols; c++)
            if ((P.lv[l].bind_mask >> c) & 1) P.bind_col[l][P.lv[l].attr[c]] = (int8_t)c;
    P.has_inl = 0;
    for (int l = 1; l < P.L; l++) {
        P.inl[l] = (P.lv[l].bind_mask == 0 && P.lv[l].key_mode == KEY_PAIR) ? 1 : 0;
        P.has_inl |= P.inl[l];
    }
    for (int l = 0; l < P.L; l++) {
        int n = l + 1;
        while (n < P.L && P.inl[n]) n++;
        P.next_lv[l] = (int8_t)n;
        int p = l - 1;
        while (p >= 0 && P.inl[p]) p--;
        P.prev_lv[l] = (int8_t)p;
    }
}

// Look up the candidate range of table `lv` for a tuple whose values are
// given by get(attr).  Returns the range size.
template <class Get>
__device__ __forceinline__ uint32_t level_lookup(const LevelDesc &lv, Get &&get, uint32_t &s, uint32_t &aux,
                                                 uint8_t &m8) {
    const int32_t k0 = get(lv.key_attr[0]);
    const int32_t k1 = lv.key_mode == KEY_PAIR ? get(lv.key_attr[1]) : 0;
    aux = 0;
    m8 = 0;
    if (lv.layout == AMJ_LAYOUT_BUCKET) {
        const uint32_t h = (lv.key_mode == KEY_PAIR ? hash_pair(k0, k1) : (uint32_t)k0) & lv.mask;
        s = lv.buc_ptrs[h];
        return lv.buc_ptrs[h + 1] - s;
    }
    const uint32_t hh = lv.key_mode == KEY_PAIR ? hash_pair(k0, k1) : hash_key(k0);
    if (lv.layout == AMJ_LAYOUT_OPEN_ADDR) {
        // run of occupied slots starting at the home slot
        uint32_t p = hh & lv.mask, len = 0;
        s = p;
        while (len <= lv.mask) {
            const int2 v = lv.slots[p];
            if (v.x == OA_EMPTY_KEY) break;
            len++;
            p = (p + 1) & lv.mask;
        }
        return len;
    }
    // cuckoo: both buckets, keep a bitmask of the slots whose key matches
    const uint32_t b1 = hh & lv.mask;
    const uint32_t b2 = (hash_key((int32_t)(hh ^ 0x5bd1e995u)) ^ 0x9e3779b9u) & lv.mask;
    uint32_t m = 0;
#pragma unroll
    for (int t = 0; t < 8; t++) {
        const uint32_t slot = t < 4 ? b1 * CUCKOO_SLOTS + t : b2 * CUCKOO_SLOTS + (t - 4);
        if (t >= 4 && b2 == b1) break;
        const int2 v = lv.slots[slot];
        const bool eq = v.x == k0 && (lv.key_mode != KEY_PAIR || v.y == k1);
        if (eq) m |= 1u << t;
    }
    s = b1;
    aux = b2;
    m8 = (uint8_t)m;
    return __popc(m);
}

// column c of candidate number `local` of an entry
__device__ __forceinline__ uint32_t candidate_slot(const LevelDesc &lv, uint32_t s, uint32_t aux, uint8_t m8,
                                                   uint32_t local) {
    if (lv.layout == AMJ_LAYOUT_BUCKET) return s + local;
    if (lv.layout == AMJ_LAYOUT_OPEN_ADDR) return (s + local) & lv.mask;
    // cuckoo: local-th set bit of m8
    uint32_t m = m8;
    for (uint32_t t = 0; t < local; t++) m &= m - 1;
    const uint32_t t = __ffs(m) - 1;
    return t < 4 ? s * CUCKOO_SLOTS + t : aux * CUCKOO_SLOTS + (t - 4);
}

__device__ __forceinline__ void load_candidate(const LevelDesc &lv, uint32_t slot, uint8_t need, int32_t *v) {
    if (lv.layout == AMJ_LAYOUT_BUCKET) {
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < lv.ncols && ((need >> c) & 1)) v[c] = lv.col[c][slot];
    } else {
        const int2 p = lv.slots[slot];
        v[0] = p.x;
        v[1] = p.y;
    }
}

}  // namespace amj
