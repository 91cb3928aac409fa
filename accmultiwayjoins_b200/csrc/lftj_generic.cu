// ALFTJ for any connected query, up to AMJ_MAX_ATTRS attributes, in any
// attribute order.  The reference's LFTJ stops at 3 attributes and 3 tables
// (LFTJ-GPU/config.h:16-17), takes 2-column relations, and binds attributes
// in the order attr_order (LFTJ-GPU/ALFTJ.cuh:1125-1196), which its driver
// always sets to the identity (LFTJ-GPU/exec_LFTJ.cu:230-231).
//
// The attributes are renamed to their positions in the order.  Every
// relation becomes a trie whose levels follow its attributes in that order
// (2 columns: build_trie2, with dense row pointers; 3 or more: build_trieN).
// An attribute at level d of a relation's trie is constrained by the list of
// values under the path of the relation's earlier attributes: level 0 is the
// whole level-0 array; deeper lists are found by descending from the root,
// one binary search per level (a dense row-pointer load at level 1).  The
// first attribute ranges over the intersection of the level-0 arrays keyed
// on it; every later one over the intersection of its lists of depth >= 1.
// The join is level-synchronous (the leapfrog of LFTJ_BFS,
// LFTJ-GPU/LFTJ_BFS.cuh:143-500, generalised): per level one count kernel
// takes, for every partial tuple, its shortest list; the candidates of all
// tuples form one space, cut into pieces of bounded size; per piece an
// expand kernel tests each candidate against the tuple's other lists
// (binary search) and either counts and hashes finished tuples (last
// attribute) or keeps survivors, which a scan compacts into the next level's
// tuples.  Memory stays bounded by the piece size whatever the intermediate
// results.  Tuples are hashed and written in attribute-id order whatever the
// binding order, so every order gives the same result.
// Lists of 2-column relations are strictly increasing (their tries drop
// repeated rows: the set semantics of the triejoin); the last level of a
// trie of 1 or of 3 or more columns keeps repeated rows, as the reference's
// IndexedTrie does (LFTJ-GPU/multi_partitioning.cuh:283-284).
#include "lftj_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

namespace amj {

constexpr int GEN_MAX_LISTS = 8;                 // relations constraining one attribute
constexpr int GEN_MAX_TRIES = 16;
constexpr uint64_t GEN_PIECE = 1ull << 26;       // candidates per expand launch

// device view of one relation's trie (2 levels with dense row pointers, or N levels)
struct GenTrie {
    const int32_t *data[TRIE_MAX_LEVELS];
    const uint64_t *off[TRIE_MAX_LEVELS - 1];
    uint64_t len0;
    TrieRef two;                                 // 2-level tries: the dense row pointers
    int levels;
};

// one list constraining an attribute: the values at level `depth` of trie
// `trie` under the path of bound attributes path[0..depth-1]
struct GenList {
    int16_t trie;
    int8_t depth;
    int8_t path[TRIE_MAX_LEVELS];
};

// the lists that constrain one attribute
struct GenLevel {
    int n;
    GenList l[GEN_MAX_LISTS];
};

struct GenArgs {
    GenLevel L;
    const GenTrie *tries;
    int level;                                   // attribute being bound (its position in the order)
    bool last;
    const int32_t *cols[AMJ_MAX_ATTRS];          // partial tuples: values of attributes 0..level-1
    uint64_t F;                                  // partial tuples
    uint8_t *sidx;                               // per tuple: its shortest list
    unsigned long long *sbeg;                    // per tuple: that list's first position
    unsigned long long *offs;                    // F + 1 exclusive candidate offsets
    uint64_t g0, g1;                             // candidate piece of this launch
    uint32_t *keep;                              // per candidate of the piece: 1 survives
    int32_t *val;                                // per candidate of the piece: its value
    unsigned long long *count, *checksum, *out_cursor;
    int32_t *out[AMJ_MAX_ATTRS];
    uint64_t out_cap;
    int k;
    int8_t opos[AMJ_MAX_ATTRS];                  // position in the order of attribute id j
};

// first index in [s, e) of base with value >= v
__device__ __forceinline__ uint64_t gen_lower(const int32_t *base, uint64_t s, uint64_t e, int32_t v) {
    while (s < e) {
        const uint64_t m = (s + e) >> 1;
        if (base[m] < v) s = m + 1;
        else e = m;
    }
    return s;
}

// range [s, e) of list i for tuple t, in the list's value array *base
__device__ __forceinline__ void gen_range(const GenArgs &A, int i, uint64_t t, const int32_t *&base, uint64_t &s,
                                          uint64_t &e) {
    const GenList &g = A.L.l[i];
    const GenTrie &T = A.tries[g.trie];
    base = T.data[g.depth];
    if (g.depth == 0) {
        s = 0;
        e = T.len0;
        return;
    }
    if (T.levels == 2) {
        child_range(T.two, A.cols[g.path[0]][t], s, e);
        return;
    }
    s = 0;
    e = T.len0;
    for (int d = 0; d < g.depth; d++) {
        const int32_t v = A.cols[g.path[d]][t];
        const uint64_t p = gen_lower(T.data[d], s, e, v);
        if (p == e || T.data[d][p] != v) {
            s = e = 0;
            return;
        }
        s = T.off[d][p];
        e = T.off[d][p + 1];
    }
}

__global__ void gen_count_kernel(const __grid_constant__ GenArgs A, unsigned long long *cnt) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < A.F; t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t best = ~0ull, bs = 0;
        int bi = 0;
        for (int i = 0; i < A.L.n; i++) {
            const int32_t *base;
            uint64_t s, e;
            gen_range(A, i, t, base, s, e);
            if (e - s < best) {
                best = e - s;
                bs = s;
                bi = i;
            }
        }
        cnt[t] = best;
        A.sidx[t] = (uint8_t)bi;
        A.sbeg[t] = bs;
    }
}

template <bool WRITE>
__global__ void gen_expand_kernel(const __grid_constant__ GenArgs A) {
    unsigned long long cnt = 0, chk = 0;
    for (uint64_t g = A.g0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < A.g1;
         g += (uint64_t)gridDim.x * blockDim.x) {
        // owner tuple: last t with offs[t] <= g
        uint64_t lo = 0, hi = A.F;
        while (hi - lo > 1) {
            const uint64_t m = (lo + hi) >> 1;
            if (A.offs[m] <= g) lo = m;
            else hi = m;
        }
        const uint64_t t = lo;
        const int si = A.sidx[t];
        const int32_t *sbase;
        uint64_t ss, se;
        gen_range(A, si, t, sbase, ss, se);
        const int32_t c = sbase[A.sbeg[t] + (g - A.offs[t])];
        bool keep = true;
        for (int i = 0; i < A.L.n && keep; i++) {
            if (i == si) continue;
            const int32_t *base;
            uint64_t s, e;
            gen_range(A, i, t, base, s, e);
            const uint64_t p = gen_lower(base, s, e, c);
            keep = p < e && base[p] == c;
        }
        if (!A.last) {
            A.keep[g - A.g0] = keep ? 1u : 0u;
            A.val[g - A.g0] = c;
            continue;
        }
        if (!keep) continue;
        // the tuple in attribute-id order: attribute j sits at position opos[j]
        uint64_t h = AMJ_CHECKSUM_SEED;
        for (int j = 0; j < A.k; j++) {
            const int l = A.opos[j];
            h = amj_hash_step(h, l == A.level ? c : A.cols[l][t]);
        }
        cnt++;
        chk += h;
        if (WRITE) {
            const unsigned long long p = atomicAdd(A.out_cursor, 1ull);
            if (p < A.out_cap)
                for (int j = 0; j < A.k; j++) {
                    const int l = A.opos[j];
                    A.out[j][p] = l == A.level ? c : A.cols[l][t];
                }
        }
    }
    if (A.last) {
        cnt = warp_sum(cnt);
        chk = warp_sum(chk);
        if ((threadIdx.x & 31) == 0 && cnt) {
            atomicAdd(A.count, cnt);
            atomicAdd(A.checksum, chk);
        }
    }
}

// survivors of a piece become the next level's tuples
__global__ void gen_compact_kernel(const __grid_constant__ GenArgs A, const uint32_t *pos, int32_t *const *ncols) {
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < A.g1 - A.g0;
         q += (uint64_t)gridDim.x * blockDim.x) {
        if (!A.keep[q]) continue;
        const uint64_t g = A.g0 + q;
        uint64_t lo = 0, hi = A.F;
        while (hi - lo > 1) {
            const uint64_t m = (lo + hi) >> 1;
            if (A.offs[m] <= g) lo = m;
            else hi = m;
        }
        const uint32_t p = pos[q];
        for (int a = 0; a < A.level; a++) ncols[a][p] = A.cols[a][lo];
        ncols[A.level][p] = A.val[q];
    }
}

struct GenQuery {
    int k = 0;
    GenLevel lv[AMJ_MAX_ATTRS];
    std::vector<Trie2> tries2;
    std::vector<TrieN> triesN;
    DBuf<GenTrie> dtries;
    int8_t opos[AMJ_MAX_ATTRS] = {};
};

struct GenRun {
    amj_ctx *ctx;
    const GenQuery *Q;
    bool write;
    int32_t *out[AMJ_MAX_ATTRS];
    uint64_t out_cap;
    DBuf<unsigned long long> ctr;   // count, checksum, out_cursor
};

static unsigned gen_grid(amj_ctx *ctx, uint64_t n) {
    const uint64_t g = (n + 255) / 256, cap = (uint64_t)ctx->num_sms * 16;
    return (unsigned)(g == 0 ? 1 : (g > cap ? cap : g));
}

// Expand the F tuples (columns cols[0..level-1]) by attribute `level`.
static int gen_expand(GenRun &R, int level, const int32_t *const *cols, uint64_t F) {
    amj_ctx *ctx = R.ctx;
    const GenQuery &Q = *R.Q;
    if (F == 0) return AMJ_OK;
    GenArgs A;
    std::memset(&A, 0, sizeof(A));
    A.L = Q.lv[level];
    A.tries = Q.dtries.p;
    A.level = level;
    A.last = level == Q.k - 1;
    A.k = Q.k;
    for (int j = 0; j < Q.k; j++) A.opos[j] = Q.opos[j];
    for (int a = 0; a < level; a++) A.cols[a] = cols[a];
    A.F = F;
    A.count = R.ctr.p;
    A.checksum = R.ctr.p + 1;
    A.out_cursor = R.ctr.p + 2;
    if (R.write) {
        for (int a = 0; a < Q.k; a++) A.out[a] = R.out[a];
        A.out_cap = R.out_cap;
    }
    DBuf<uint8_t> sidx;
    DBuf<unsigned long long> sbeg, offs;
    AMJ_TRY(sidx.alloc(ctx, F));
    AMJ_TRY(sbeg.alloc(ctx, F));
    AMJ_TRY(offs.alloc(ctx, F + 1));
    A.sidx = sidx.p;
    A.sbeg = sbeg.p;
    A.offs = offs.p;
    note_launch(ctx);
    gen_count_kernel<<<gen_grid(ctx, F), 256, 0, ctx->stream>>>(A, offs.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_TRY(scan_exclusive_u64(ctx, (const uint64_t *)offs.p, (uint64_t *)offs.p, F, (uint64_t *)offs.p + F));
    unsigned long long T = 0;
    AMJ_CUDA_TRY(cudaMemcpyAsync(&T, offs.p + F, 8, cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (uint64_t g0 = 0; g0 < T; g0 += GEN_PIECE) {
        A.g0 = g0;
        A.g1 = std::min<uint64_t>(T, g0 + GEN_PIECE);
        const uint64_t P = A.g1 - A.g0;
        if (A.last) {
            note_launch(ctx);
            if (R.write) gen_expand_kernel<true><<<gen_grid(ctx, P), 256, 0, ctx->stream>>>(A);
            else gen_expand_kernel<false><<<gen_grid(ctx, P), 256, 0, ctx->stream>>>(A);
            AMJ_CUDA_TRY(cudaGetLastError());
            continue;
        }
        DBuf<uint32_t> keep, pos;
        DBuf<int32_t> val;
        AMJ_TRY(keep.alloc(ctx, P));
        AMJ_TRY(pos.alloc(ctx, P + 1));
        AMJ_TRY(val.alloc(ctx, P));
        A.keep = keep.p;
        A.val = val.p;
        note_launch(ctx);
        gen_expand_kernel<false><<<gen_grid(ctx, P), 256, 0, ctx->stream>>>(A);
        AMJ_CUDA_TRY(cudaGetLastError());
        AMJ_TRY(scan_exclusive_u32(ctx, keep.p, pos.p, P, pos.p + P));
        uint32_t nf = 0;
        AMJ_CUDA_TRY(cudaMemcpyAsync(&nf, pos.p + P, 4, cudaMemcpyDeviceToHost, ctx->stream));
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (nf == 0) continue;
        std::vector<DBuf<int32_t>> nbuf(level + 1);
        int32_t *ncols[AMJ_MAX_ATTRS] = {};
        for (int a = 0; a <= level; a++) {
            AMJ_TRY(nbuf[a].alloc(ctx, nf));
            ncols[a] = nbuf[a].p;
        }
        DBuf<int32_t *> dcols;
        AMJ_TRY(dcols.alloc(ctx, level + 1));
        AMJ_CUDA_TRY(cudaMemcpyAsync(dcols.p, ncols, (level + 1) * sizeof(int32_t *), cudaMemcpyHostToDevice,
                                     ctx->stream));
        note_launch(ctx);
        gen_compact_kernel<<<gen_grid(ctx, P), 256, 0, ctx->stream>>>(A, pos.p, dcols.p);
        AMJ_CUDA_TRY(cudaGetLastError());
        keep.release();
        val.release();
        pos.release();
        AMJ_TRY(gen_expand(R, level + 1, ncols, nf));
    }
    return AMJ_OK;
}

// One pass of the whole join: count and checksum, and the tuples with `out`.
static int gen_pass(amj_ctx *ctx, const GenQuery &Q, int32_t *const *out, uint64_t out_cap, uint64_t *count,
                    uint64_t *checksum, uint64_t *written) {
    GenRun R{ctx, &Q, out != nullptr, {}, out_cap, {}};
    if (out)
        for (int a = 0; a < Q.k; a++) R.out[a] = out[a];
    AMJ_TRY(R.ctr.alloc(ctx, 3));
    AMJ_CUDA_TRY(cudaMemsetAsync(R.ctr.p, 0, 3 * sizeof(unsigned long long), ctx->stream));
    // level 0 is the expansion of one empty tuple by the level-0 arrays
    AMJ_TRY(gen_expand(R, 0, nullptr, 1));
    unsigned long long h[3];
    AMJ_CUDA_TRY(cudaMemcpyAsync(h, R.ctr.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_TRY(status_check(ctx, "LFTJ generic"));
    *count = h[0];
    *checksum = h[1];
    if (written) *written = std::min<unsigned long long>(h[2], out_cap);
    return AMJ_OK;
}

// The compiled query without tries: positions in the binding order, every
// relation's columns in that order, and the lists that constrain each
// attribute (list i of level l refers to relation trie).
struct GenPlan {
    int k = 0;
    int nrels = 0;
    int pos[AMJ_MAX_ATTRS] = {};
    int ncols[GEN_MAX_TRIES] = {};
    int colord[GEN_MAX_TRIES][TRIE_MAX_LEVELS] = {};
    GenLevel lv[AMJ_MAX_ATTRS];
};

// Plan a query: attributes 0..k-1, bound in the order `order` (null: the
// identity); every attribute after the first in the order must share a
// relation with an earlier one.
static int gen_plan(amj_rel *const *rels, int nrels, const uint32_t *order, GenPlan *P) {
    if (nrels > GEN_MAX_TRIES) return fail(AMJ_EUNSUPPORTED, "LFTJ: at most 16 relations");
    uint32_t seen = 0;
    for (int i = 0; i < nrels; i++) {
        if (rels[i]->ncols < 1 || rels[i]->ncols > TRIE_MAX_LEVELS)
            return fail(AMJ_EUNSUPPORTED, "LFTJ: relations of 1 to 8 columns");
        uint32_t mine = 0;
        for (int c = 0; c < rels[i]->ncols; c++) {
            if (rels[i]->attrs[c] >= 32 || ((mine >> rels[i]->attrs[c]) & 1))
                return fail(AMJ_EINVAL, "LFTJ: a relation repeats an attribute");
            mine |= 1u << rels[i]->attrs[c];
        }
        seen |= mine;
    }
    int k = 0;
    while (k < 32 && ((seen >> k) & 1)) k++;
    if (seen != ((1u << k) - 1) || k > AMJ_MAX_ATTRS)
        return fail(AMJ_EINVAL, "LFTJ: the relations' attributes must be exactly 0..k-1 with k <= 8");
    P->k = k;
    P->nrels = nrels;
    int *pos = P->pos;
    for (int a = 0; a < k; a++) pos[a] = -1;
    for (int i = 0; i < k; i++) {
        const uint32_t a = order ? order[i] : (uint32_t)i;
        if (a >= (uint32_t)k || pos[a] >= 0)
            return fail(AMJ_EINVAL, "LFTJ: the attribute order must be a permutation of 0..k-1");
        pos[a] = i;
    }
    for (int l = 0; l < k; l++) P->lv[l].n = 0;
    for (int i = 0; i < nrels; i++) {
        // the relation's columns in binding order
        const int nc = rels[i]->ncols;
        P->ncols[i] = nc;
        int *colord = P->colord[i];
        for (int c = 0; c < nc; c++) colord[c] = c;
        std::sort(colord, colord + nc, [&](int x, int y) { return pos[rels[i]->attrs[x]] < pos[rels[i]->attrs[y]]; });
        // one list per attribute at depth >= 1; a level-0 list for the first
        // attribute, and for a 1-column relation (nothing deeper implies it)
        for (int d = 0; d < nc; d++) {
            const int l = pos[rels[i]->attrs[colord[d]]];
            if (d == 0 && l != 0 && nc > 1) continue;
            GenLevel &L = P->lv[l];
            if (L.n >= GEN_MAX_LISTS) return fail(AMJ_EUNSUPPORTED, "LFTJ: more than 8 relations constrain one attribute");
            GenList &gl = L.l[L.n++];
            std::memset(&gl, 0, sizeof(gl));
            gl.trie = (int16_t)i;
            gl.depth = (int8_t)d;
            for (int e = 0; e < d; e++) gl.path[e] = (int8_t)pos[rels[i]->attrs[colord[e]]];
        }
    }
    for (int l = 1; l < k; l++) {
        bool linked = false;
        for (int j = 0; j < P->lv[l].n; j++) linked |= P->lv[l].l[j].depth > 0;
        if (!linked)
            return fail(AMJ_EUNSUPPORTED, "LFTJ: every attribute after the first must share a relation with an earlier one");
    }
    if (P->lv[0].n == 0) return fail(AMJ_EUNSUPPORTED, "LFTJ: no relation starts with the first attribute");
    return AMJ_OK;
}

static void gen_query_from_plan(const GenPlan &P, GenQuery *Q) {
    Q->k = P.k;
    for (int l = 0; l < P.k; l++) Q->lv[l] = P.lv[l];
    for (int a = 0; a < P.k && a < AMJ_MAX_ATTRS; a++) Q->opos[a] = (int8_t)P.pos[a];
}

// The trie of relation i in its binding column order, on the device.
static int gen_build_trie(amj_ctx *ctx, const amj_rel *r, const GenPlan &P, int i, Trie2 *t2, TrieN *tn,
                          GenTrie *g) {
    const int nc = P.ncols[i];
    const int *colord = P.colord[i];
    std::memset(g, 0, sizeof(*g));
    if (nc == 2) {
        AMJ_TRY(build_trie2(ctx, r->d_cols[colord[0]], r->d_cols[colord[1]], r->n, t2, true));
        g->levels = 2;
        g->data[0] = t2->data0.p;
        g->data[1] = t2->data1.p;
        g->off[0] = t2->off0.p;
        g->len0 = t2->len0;
        g->two = trie_ref(*t2);
        return AMJ_OK;
    }
    const int32_t *cols[TRIE_MAX_LEVELS];
    for (int c = 0; c < nc; c++) cols[c] = r->d_cols[colord[c]];
    AMJ_TRY(build_trieN(ctx, cols, nc, r->n, tn));
    g->levels = nc;
    for (int c = 0; c < nc; c++) g->data[c] = tn->data[c].p;
    for (int c = 0; c + 1 < nc; c++) g->off[c] = tn->off[c].p;
    g->len0 = tn->len[0];
    return AMJ_OK;
}

int lftj_generic_compile(amj_ctx *ctx, amj_rel *const *rels, int nrels, const uint32_t *order, GenQuery *Q) {
    GenPlan P;
    AMJ_TRY(gen_plan(rels, nrels, order, &P));
    for (int i = 0; i < nrels; i++)
        if (rels[i]->where == AMJ_MEM_HOST_STREAMED)
            return fail(AMJ_EUNSUPPORTED, "LFTJ: host-resident relations need ooc = 1");
    gen_query_from_plan(P, Q);
    std::vector<GenTrie> ht(nrels);
    Q->tries2.resize(nrels);
    Q->triesN.resize(nrels);
    for (int i = 0; i < nrels; i++) AMJ_TRY(gen_build_trie(ctx, rels[i], P, i, &Q->tries2[i], &Q->triesN[i], &ht[i]));
    AMJ_TRY(Q->dtries.alloc(ctx, nrels));
    AMJ_CUDA_TRY(cudaMemcpyAsync(Q->dtries.p, ht.data(), nrels * sizeof(GenTrie), cudaMemcpyHostToDevice, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return AMJ_OK;
}

// ---- out-of-core ----
// The reference's OOCWrapper (LFTJ-GPU/ooc_wrapper.cuh:14-427) splits a
// memory budget over the attributes in proportion to the tries each one
// heads (BudgetPlanner, :14-49), chooses for every such attribute value
// ranges of the heading tries' level 0 whose sub-tries fit its share (probe,
// :110-172), provisions the trie slices of each combination of ranges
// (:68-104) and joins every combination (:263-371); the ranges of one
// attribute partition its values, so every result tuple is found in exactly
// one combination.  Here the tries live in pinned host memory: a relation on
// the device has its trie built there and copied out; a host-resident
// relation (AMJ_MEM_HOST_STREAMED) is cut into value ranges of its first
// column (in binding order) that fit the budget, and the trie of each range
// is built on the device and appended (the ranges come in increasing order,
// so the appended tries are the trie of the whole relation).  Each
// combination copies to the device only the slices that changed since the
// previous one, rebases their offsets and runs the generic join over them.

struct HostTrie {
    int levels = 0;
    uint64_t len[TRIE_MAX_LEVELS] = {};
    int32_t *data[TRIE_MAX_LEVELS] = {};    // pinned
    uint64_t *off[TRIE_MAX_LEVELS - 1] = {};
    HostTrie() = default;
    HostTrie(const HostTrie &) = delete;
    HostTrie &operator=(const HostTrie &) = delete;
    ~HostTrie() {
        for (auto *p : data)
            if (p) cudaFreeHost(p);
        for (auto *p : off)
            if (p) cudaFreeHost(p);
    }
    // entry ranges [s[l], e[l]) of every level for level-0 entries [i0, i1)
    void ranges(uint64_t i0, uint64_t i1, uint64_t *s, uint64_t *e) const {
        s[0] = i0;
        e[0] = i1;
        for (int l = 0; l + 1 < levels; l++) {
            s[l + 1] = off[l][s[l]];
            e[l + 1] = off[l][e[l]];
        }
    }
    uint64_t bytes(uint64_t i0, uint64_t i1) const {
        uint64_t s[TRIE_MAX_LEVELS], e[TRIE_MAX_LEVELS];
        ranges(i0, i1, s, e);
        uint64_t b = 0;
        for (int l = 0; l < levels; l++) b += 4 * (e[l] - s[l]) + (l + 1 < levels ? 8 * (e[l] - s[l] + 1) : 0);
        return b;
    }
    // level-0 entries whose values lie in [lo, hi]
    void value_range(int64_t lo, int64_t hi, uint64_t *i0, uint64_t *i1) const {
        const int32_t *d = data[0];
        *i0 = (uint64_t)(std::lower_bound(d, d + len[0], (int64_t)lo, [](int32_t a, int64_t v) { return a < v; }) - d);
        *i1 = (uint64_t)(std::upper_bound(d, d + len[0], (int64_t)hi, [](int64_t v, int32_t a) { return v < a; }) - d);
    }
};

static int host_alloc(void **p, size_t bytes) {
    if (cudaMallocHost(p, bytes ? bytes : 4) != cudaSuccess) {
        (void)cudaGetLastError();
        *p = nullptr;
        return fail(AMJ_ENOMEM, "LFTJ ooc: pinned host allocation failed");
    }
    return AMJ_OK;
}

// Append the device trie g (levels nc) to the host trie H.
static int append_trie(amj_ctx *ctx, const GenTrie &g, const uint64_t *lens, HostTrie *H, uint64_t *cap) {
    // grow the pinned arrays when needed (doubling)
    for (int l = 0; l < H->levels; l++) {
        const uint64_t need = H->len[l] + lens[l];
        if (need > cap[l]) {
            uint64_t nc = std::max<uint64_t>(need, cap[l] * 2);
            void *nd = nullptr, *no = nullptr;
            AMJ_TRY(host_alloc(&nd, nc * 4));
            if (H->data[l]) std::memcpy(nd, H->data[l], H->len[l] * 4);
            if (H->data[l]) cudaFreeHost(H->data[l]);
            H->data[l] = (int32_t *)nd;
            if (l + 1 < H->levels) {
                AMJ_TRY(host_alloc(&no, (nc + 1) * 8));
                if (H->off[l]) std::memcpy(no, H->off[l], (H->len[l] + 1) * 8);
                else ((uint64_t *)no)[0] = 0;
                if (H->off[l]) cudaFreeHost(H->off[l]);
                H->off[l] = (uint64_t *)no;
            }
            cap[l] = nc;
        }
    }
    for (int l = 0; l < H->levels; l++) {
        if (lens[l])
            AMJ_CUDA_TRY(cudaMemcpyAsync(H->data[l] + H->len[l], g.data[l], lens[l] * 4, cudaMemcpyDeviceToHost,
                                         ctx->stream));
        if (l + 1 < H->levels)
            AMJ_CUDA_TRY(cudaMemcpyAsync(H->off[l] + H->len[l], g.off[l], (lens[l] + 1) * 8, cudaMemcpyDeviceToHost,
                                         ctx->stream));
    }
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    // the appended offsets continue from the next level's previous end
    for (int l = 0; l + 1 < H->levels; l++) {
        const uint64_t base = H->len[l + 1];
        for (uint64_t j = 0; j <= lens[l]; j++) H->off[l][H->len[l] + j] += base;
    }
    for (int l = 0; l < H->levels; l++) H->len[l] += lens[l];
    return AMJ_OK;
}

// The host trie of relation i (columns in binding order), built in ranges of
// its first column's values that keep each range's rows within `budget`
// bytes of device memory.
static int build_host_trie(amj_ctx *ctx, const amj_rel *r, const GenPlan &P, int i, uint64_t budget, HostTrie *H) {
    const int nc = P.ncols[i];
    H->levels = nc;
    uint64_t cap[TRIE_MAX_LEVELS] = {};
    for (int l = 0; l < nc; l++) {
        void *d = nullptr;
        AMJ_TRY(host_alloc(&d, 4));
        H->data[l] = (int32_t *)d;
        cap[l] = 1;
        if (l + 1 < nc) {
            void *o = nullptr;
            AMJ_TRY(host_alloc(&o, 16));
            H->off[l] = (uint64_t *)o;
            H->off[l][0] = 0;
        }
    }
    auto add = [&](const int32_t *const *dcols, uint64_t n) -> int {
        amj_rel view;
        view.ctx = ctx;
        view.n = n;
        view.ncols = nc;
        for (int c = 0; c < nc; c++) {
            view.attrs[c] = (uint32_t)c;
            view.d_cols[c] = const_cast<int32_t *>(dcols[c]);
        }
        GenPlan one;
        one.ncols[0] = nc;
        for (int c = 0; c < nc; c++) one.colord[0][c] = c;
        Trie2 t2;
        TrieN tn;
        GenTrie g;
        AMJ_TRY(gen_build_trie(ctx, &view, one, 0, &t2, &tn, &g));
        uint64_t lens[TRIE_MAX_LEVELS] = {};
        if (nc == 2) {
            lens[0] = t2.len0;
            lens[1] = t2.len1;
        } else {
            for (int l = 0; l < nc; l++) lens[l] = tn.len[l];
        }
        return append_trie(ctx, g, lens, H, cap);
    };
    if (r->where != AMJ_MEM_HOST_STREAMED) {
        const int32_t *cols[TRIE_MAX_LEVELS];
        for (int c = 0; c < nc; c++) cols[c] = r->d_cols[P.colord[i][c]];
        return add(cols, r->n);
    }
    // a host-resident relation: value ranges of its first column, each range's
    // rows gathered on the host, copied, built and appended in increasing order
    const int32_t *h0 = r->h_cols[P.colord[i][0]];
    const uint64_t n = r->n;
    if (n == 0) return AMJ_OK;
    int64_t vmin = INT32_MAX, vmax = INT32_MIN;
#pragma omp parallel for reduction(min : vmin) reduction(max : vmax)
    for (int64_t j = 0; j < (int64_t)n; j++) {
        vmin = std::min<int64_t>(vmin, h0[j]);
        vmax = std::max<int64_t>(vmax, h0[j]);
    }
    // rows per range: the sort and the trie take about 40 bytes a row
    const uint64_t per = std::max<uint64_t>(1024, budget / (uint64_t)(40 + 8 * nc));
    const uint64_t parts = std::max<uint64_t>(1, (n + per - 1) / per);
    // value boundaries from a histogram of 4096 buckets over [vmin, vmax]
    const int NB = 4096;
    const double width = ((double)vmax - (double)vmin + 1.0) / NB;
    std::vector<uint64_t> hist(NB, 0);
    for (uint64_t j = 0; j < n; j++) hist[std::min<int64_t>(NB - 1, (int64_t)(((double)h0[j] - (double)vmin) / width))]++;
    std::vector<int64_t> bounds;   // exclusive upper value bounds of the ranges
    uint64_t acc = 0;
    const uint64_t target = (n + parts - 1) / parts;
    for (int b = 0; b < NB; b++) {
        acc += hist[b];
        if (acc >= target && b + 1 < NB) {
            bounds.push_back(vmin + (int64_t)std::ceil((b + 1) * width));
            acc = 0;
        }
    }
    bounds.push_back(vmax + 1);
    // one pass puts every row in its range (bounds ascending)
    const size_t R = bounds.size();
    std::vector<std::vector<std::vector<int32_t>>> part(R, std::vector<std::vector<int32_t>>(nc));
    for (uint64_t j = 0; j < n; j++) {
        const size_t q = (size_t)(std::upper_bound(bounds.begin(), bounds.end(), (int64_t)h0[j]) - bounds.begin());
        for (int c = 0; c < nc; c++) part[q][c].push_back(r->h_cols[P.colord[i][c]][j]);
    }
    for (size_t q = 0; q < R; q++) {
        std::vector<std::vector<int32_t>> hc = std::move(part[q]);
        const uint64_t m = hc[0].size();
        if (m == 0) continue;
        std::vector<DBuf<int32_t>> dc(nc);
        const int32_t *cols[TRIE_MAX_LEVELS];
        for (int c = 0; c < nc; c++) {
            AMJ_TRY(dc[c].alloc(ctx, m));
            AMJ_CUDA_TRY(cudaMemcpyAsync(dc[c].p, hc[c].data(), m * 4, cudaMemcpyHostToDevice, ctx->stream));
            cols[c] = dc[c].p;
        }
        AMJ_TRY(add(cols, m));
    }
    return AMJ_OK;
}

__global__ void rebase_offsets_kernel(uint64_t *off, uint64_t n, uint64_t base) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        off[i] -= base;
}

// The device copy of one trie's slice (level-0 entries [i0, i1)).
struct DevSlice {
    uint64_t i0 = ~0ull, i1 = ~0ull;   // the slice the buffers hold
    uint64_t cap[TRIE_MAX_LEVELS] = {};
    DBuf<int32_t> data[TRIE_MAX_LEVELS];
    DBuf<uint64_t> off[TRIE_MAX_LEVELS - 1];
};

static int provision(amj_ctx *ctx, const HostTrie &H, uint64_t i0, uint64_t i1, DevSlice *S, GenTrie *g,
                     uint64_t *copied) {
    uint64_t s[TRIE_MAX_LEVELS], e[TRIE_MAX_LEVELS];
    H.ranges(i0, i1, s, e);
    if (S->i0 != i0 || S->i1 != i1) {
        for (int l = 0; l < H.levels; l++) {
            const uint64_t m = e[l] - s[l];
            if (m + TRIE_LEVEL1_PAD > S->cap[l]) {
                S->cap[l] = std::max<uint64_t>(m + TRIE_LEVEL1_PAD, S->cap[l] * 3 / 2);
                AMJ_TRY(S->data[l].alloc(ctx, S->cap[l]));
                if (l + 1 < H.levels) AMJ_TRY(S->off[l].alloc(ctx, S->cap[l] + 1));
            }
            if (m) AMJ_CUDA_TRY(cudaMemcpyAsync(S->data[l].p, H.data[l] + s[l], m * 4, cudaMemcpyHostToDevice,
                                                ctx->stream));
            *copied += 4 * m;
            if (l + 1 < H.levels) {
                AMJ_CUDA_TRY(cudaMemcpyAsync(S->off[l].p, H.off[l] + s[l], (m + 1) * 8, cudaMemcpyHostToDevice,
                                             ctx->stream));
                *copied += 8 * (m + 1);
                const uint64_t base = H.off[l][s[l]];
                if (base) {
                    note_launch(ctx);
                    rebase_offsets_kernel<<<gen_grid(ctx, m + 1), 256, 0, ctx->stream>>>(S->off[l].p, m + 1, base);
                    AMJ_CUDA_TRY(cudaGetLastError());
                }
            }
        }
        S->i0 = i0;
        S->i1 = i1;
    }
    std::memset(g, 0, sizeof(*g));
    g->levels = H.levels;
    for (int l = 0; l < H.levels; l++) g->data[l] = S->data[l].p;
    for (int l = 0; l + 1 < H.levels; l++) g->off[l] = S->off[l].p;
    g->len0 = i1 - i0;
    if (H.levels == 2) {
        g->two.data0 = g->data[0];
        g->two.off0 = g->off[0];
        g->two.data1 = g->data[1];
        g->two.len0 = g->len0;
        g->two.rp_count = 0;   // no dense row pointers: child lists by binary search
    }
    return AMJ_OK;
}

int lftj_generic_ooc_execute(amj_ctx *ctx, amj_rel *const *rels, int nrels, int flags, const uint32_t *order,
                             amj_result *out) {
    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1], e2 = ctx->ev[2];
    AMJ_CUDA_TRY(cudaEventRecord(e0, ctx->stream));
    GenPlan P;
    AMJ_TRY(gen_plan(rels, nrels, order, &P));
    result_init(out, P.k);
    uint64_t budget = ctx->opts.mem_budget;
    if (!budget) {
        size_t fr = 0, tot = 0;
        AMJ_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        budget = fr / 2;
    }
    // host tries, one per distinct (relation, column order)
    std::vector<std::unique_ptr<HostTrie>> hosts;
    std::vector<int> host_of(nrels, -1);
    for (int i = 0; i < nrels; i++) {
        for (int j = 0; j < i && host_of[i] < 0; j++)
            if (rels[j] == rels[i] || (rels[j]->d_cols[0] == rels[i]->d_cols[0] && rels[j]->h_cols[0] == rels[i]->h_cols[0] &&
                                       rels[j]->n == rels[i]->n && P.ncols[j] == P.ncols[i])) {
                bool same = true;
                for (int c = 0; c < P.ncols[i]; c++)
                    same &= rels[j]->d_cols[P.colord[j][c]] == rels[i]->d_cols[P.colord[i][c]] &&
                            rels[j]->h_cols[P.colord[j][c]] == rels[i]->h_cols[P.colord[i][c]];
                if (same) host_of[i] = host_of[j];
            }
        if (host_of[i] >= 0) continue;
        hosts.emplace_back(new HostTrie());
        host_of[i] = (int)hosts.size() - 1;
        AMJ_TRY(build_host_trie(ctx, rels[i], P, i, budget, hosts.back().get()));
    }
    AMJ_CUDA_TRY(cudaEventRecord(e1, ctx->stream));
    // the tries each attribute heads (level 0 in binding order), and the
    // budget share of each attribute: in proportion to its tries
    std::vector<std::vector<int>> heads(P.k);
    for (int i = 0; i < nrels; i++) heads[P.pos[rels[i]->attrs[P.colord[i][0]]]].push_back(i);
    // value ranges per heading attribute: the longest ranges whose heading
    // slices fit the share (at least one value per range)
    std::vector<std::vector<std::pair<int64_t, int64_t>>> ranges(P.k);
    for (int l = 0; l < P.k; l++) {
        if (heads[l].empty()) continue;
        const uint64_t share = std::max<uint64_t>(1, budget / (uint64_t)nrels * heads[l].size());
        int64_t vmin = INT64_MAX, vmax = INT64_MIN;
        for (int i : heads[l]) {
            const HostTrie &H = *hosts[host_of[i]];
            if (H.len[0]) {
                vmin = std::min<int64_t>(vmin, H.data[0][0]);
                vmax = std::max<int64_t>(vmax, H.data[0][H.len[0] - 1]);
            }
        }
        if (vmin > vmax) {   // every heading trie is empty: no result
            ranges.assign(P.k, {});
            break;
        }
        auto fits = [&](int64_t lo, int64_t hi) {
            uint64_t b = 0;
            for (int i : heads[l]) {
                const HostTrie &H = *hosts[host_of[i]];
                uint64_t i0, i1;
                H.value_range(lo, hi, &i0, &i1);
                b += H.bytes(i0, i1);
            }
            return b <= share;
        };
        int64_t lo = vmin;
        while (lo <= vmax) {
            int64_t a = lo, b = vmax;   // the largest hi in [lo, vmax] that fits (at least lo)
            if (fits(lo, vmax)) a = vmax;
            else
                while (a < b) {
                    const int64_t m = a + (b - a + 1) / 2;
                    if (fits(lo, m)) a = m;
                    else b = m - 1;
                }
            ranges[l].push_back({lo, a});
            lo = a + 1;
        }
    }
    // the combinations: one range per heading attribute (odometer order, the
    // deepest attribute fastest, so the slices of the outer ones stay)
    std::vector<int> lvls;
    for (int l = 0; l < P.k; l++)
        if (!heads[l].empty()) lvls.push_back(l);
    bool empty = false;
    for (int l : lvls) empty |= ranges[l].empty();
    // relations over the same host trie and heading attribute share one
    // device slice (the views of a self-join)
    std::vector<int> slot(nrels);
    for (int i = 0; i < nrels; i++) {
        slot[i] = i;
        const int li = P.pos[rels[i]->attrs[P.colord[i][0]]];
        for (int j = 0; j < i; j++)
            if (host_of[j] == host_of[i] && P.pos[rels[j]->attrs[P.colord[j][0]]] == li) {
                slot[i] = slot[j];
                break;
            }
    }
    GenQuery Q;
    gen_query_from_plan(P, &Q);
    AMJ_TRY(Q.dtries.alloc(ctx, nrels));
    std::vector<DevSlice> slices(nrels);
    std::vector<GenTrie> ht(nrels);
    std::vector<size_t> idx(lvls.size(), 0);
    const bool materialize = (flags & AMJ_F_MATERIALIZE) != 0;
    std::vector<std::vector<int32_t>> hcols(materialize ? P.k : 0);
    uint64_t count = 0, checksum = 0, combos = 0, copied = 0;
    while (!empty) {
        for (size_t j = 0; j < lvls.size(); j++) {
            const auto rg = ranges[lvls[j]][idx[j]];
            for (int i : heads[lvls[j]]) {
                if (slot[i] != i) continue;
                const HostTrie &H = *hosts[host_of[i]];
                uint64_t i0, i1;
                H.value_range(rg.first, rg.second, &i0, &i1);
                AMJ_TRY(provision(ctx, H, i0, i1, &slices[i], &ht[i], &copied));
            }
        }
        for (int i = 0; i < nrels; i++) ht[i] = ht[slot[i]];
        AMJ_CUDA_TRY(cudaMemcpyAsync(Q.dtries.p, ht.data(), nrels * sizeof(GenTrie), cudaMemcpyHostToDevice, ctx->stream));
        uint64_t c = 0, h = 0;
        AMJ_TRY(gen_pass(ctx, Q, nullptr, 0, &c, &h, nullptr));
        if (materialize && c) {
            std::vector<DBuf<int32_t>> dc(P.k);
            int32_t *cols[AMJ_MAX_ATTRS] = {};
            for (int a = 0; a < P.k; a++) {
                AMJ_TRY(dc[a].alloc(ctx, c));
                cols[a] = dc[a].p;
            }
            uint64_t c2 = 0, h2 = 0, w = 0;
            AMJ_TRY(gen_pass(ctx, Q, cols, c, &c2, &h2, &w));
            if (c2 != c || h2 != h || w != c) return fail(AMJ_ECUDA, "LFTJ ooc: write pass disagrees with count pass");
            for (int a = 0; a < P.k; a++) {
                const size_t old = hcols[a].size();
                hcols[a].resize(old + c);
                AMJ_CUDA_TRY(cudaMemcpyAsync(hcols[a].data() + old, cols[a], c * 4, cudaMemcpyDeviceToHost, ctx->stream));
            }
            AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        }
        count += c;
        checksum += h;
        combos++;
        // next combination
        int j = (int)lvls.size() - 1;
        while (j >= 0 && ++idx[j] == ranges[lvls[j]].size()) idx[j--] = 0;
        if (j < 0) break;
    }
    out->count = count;
    out->checksum = checksum;
    out->stats[7] = combos;     // slice combinations joined
    if (materialize) {
        auto *o = new ResultOwner();
        o->ctx = ctx;
        out->priv = o;
        out->rows = count;
        out->on_host = 1;
        for (int a = 0; a < P.k; a++) {
            if (cudaMallocHost((void **)&out->cols[a], (count ? count : 1) * 4) != cudaSuccess) {
                (void)cudaGetLastError();
                amj_result_release(out);
                return fail(AMJ_ENOMEM, "LFTJ ooc: pinned result allocation failed");
            }
            if (count) std::memcpy(out->cols[a], hcols[a].data(), count * 4);
        }
    }
    AMJ_CUDA_TRY(cudaEventRecord(e2, ctx->stream));
    AMJ_CUDA_TRY(cudaEventSynchronize(e2));
    out->build_ms = event_ms(e0, e1);
    out->probe_ms = event_ms(e1, e2);
    out->total_ms = event_ms(e0, e2);
    if (materialize) {
        const int rc = finish_result_columns(ctx, out, flags);
        if (rc != AMJ_OK) {
            amj_result_release(out);
            return rc;
        }
    }
    return AMJ_OK;
}

// amj_lftj_execute for queries other than the triangle: a count pass, then
// with AMJ_F_MATERIALIZE a write pass into exactly allocated columns.
int lftj_generic_execute(amj_ctx *ctx, amj_rel *const *rels, int nrels, int ooc, int flags, const uint32_t *order,
                         amj_result *out) {
    if (ooc) return lftj_generic_ooc_execute(ctx, rels, nrels, flags, order, out);
    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1], e2 = ctx->ev[2];
    AMJ_CUDA_TRY(cudaEventRecord(e0, ctx->stream));
    GenQuery Q;
    AMJ_TRY(lftj_generic_compile(ctx, rels, nrels, order, &Q));
    result_init(out, Q.k);
    AMJ_CUDA_TRY(cudaEventRecord(e1, ctx->stream));
    uint64_t c = 0, h = 0;
    AMJ_TRY(gen_pass(ctx, Q, nullptr, 0, &c, &h, nullptr));
    out->count = c;
    out->checksum = h;
    const bool materialize = (flags & AMJ_F_MATERIALIZE) != 0;
    if (materialize) {
        int32_t *cols[AMJ_MAX_ATTRS] = {};
        int rc = AMJ_OK;
        for (int a = 0; a < Q.k && rc == AMJ_OK; a++) rc = dev_alloc(ctx, (void **)&cols[a], (c ? c : 1) * 4);
        uint64_t c2 = 0, h2 = 0, w = 0;
        if (rc == AMJ_OK) rc = gen_pass(ctx, Q, cols, c, &c2, &h2, &w);
        if (rc == AMJ_OK && (c2 != c || h2 != h || w != c))
            rc = fail(AMJ_ECUDA, "LFTJ generic: write pass disagrees with count pass");
        if (rc != AMJ_OK) {
            for (int a = 0; a < Q.k; a++) dev_free(ctx, cols[a]);
            return rc;
        }
        auto *o = new ResultOwner();
        o->ctx = ctx;
        out->priv = o;
        out->rows = c;
        for (int a = 0; a < Q.k; a++) out->cols[a] = cols[a];
    }
    AMJ_CUDA_TRY(cudaEventRecord(e2, ctx->stream));
    AMJ_CUDA_TRY(cudaEventSynchronize(e2));
    out->build_ms = event_ms(e0, e1);
    out->probe_ms = event_ms(e1, e2);
    out->total_ms = event_ms(e0, e2);
    if (materialize) {
        const int rc = finish_result_columns(ctx, out, flags);
        if (rc != AMJ_OK) {
            amj_result_release(out);
            return rc;
        }
    }
    return AMJ_OK;
}

}  // namespace amj
