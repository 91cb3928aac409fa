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
#include <cstring>
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

// Compile a query: attributes 0..k-1, bound in the order `order` (null: the
// identity); every attribute after the first in the order must share a
// relation with an earlier one.
int lftj_generic_compile(amj_ctx *ctx, amj_rel *const *rels, int nrels, const uint32_t *order, GenQuery *Q) {
    if (nrels > GEN_MAX_TRIES) return fail(AMJ_EUNSUPPORTED, "LFTJ: at most 16 relations");
    uint32_t seen = 0;
    for (int i = 0; i < nrels; i++) {
        if (rels[i]->ncols < 1 || rels[i]->ncols > TRIE_MAX_LEVELS)
            return fail(AMJ_EUNSUPPORTED, "LFTJ: relations of 1 to 8 columns");
        if (rels[i]->where == AMJ_MEM_HOST_STREAMED)
            return fail(AMJ_EUNSUPPORTED, "LFTJ: relations must be on the device");
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
    Q->k = k;
    // position of every attribute in the binding order
    int pos[AMJ_MAX_ATTRS];
    for (int a = 0; a < k; a++) pos[a] = -1;
    for (int i = 0; i < k; i++) {
        const uint32_t a = order ? order[i] : (uint32_t)i;
        if (a >= (uint32_t)k || pos[a] >= 0)
            return fail(AMJ_EINVAL, "LFTJ: the attribute order must be a permutation of 0..k-1");
        pos[a] = i;
    }
    for (int a = 0; a < k && a < AMJ_MAX_ATTRS; a++) Q->opos[a] = (int8_t)pos[a];
    for (int l = 0; l < k; l++) Q->lv[l].n = 0;
    std::vector<GenTrie> ht(nrels);
    Q->tries2.resize(nrels);
    Q->triesN.resize(nrels);
    for (int i = 0; i < nrels; i++) {
        // the relation's columns in binding order
        const int nc = rels[i]->ncols;
        int colord[TRIE_MAX_LEVELS];
        for (int c = 0; c < nc; c++) colord[c] = c;
        std::sort(colord, colord + nc, [&](int x, int y) { return pos[rels[i]->attrs[x]] < pos[rels[i]->attrs[y]]; });
        GenTrie &g = ht[i];
        std::memset(&g, 0, sizeof(g));
        if (nc == 2) {
            AMJ_TRY(build_trie2(ctx, rels[i]->d_cols[colord[0]], rels[i]->d_cols[colord[1]], rels[i]->n,
                                &Q->tries2[i], true));
            const Trie2 &t = Q->tries2[i];
            g.levels = 2;
            g.data[0] = t.data0.p;
            g.data[1] = t.data1.p;
            g.off[0] = t.off0.p;
            g.len0 = t.len0;
            g.two = trie_ref(t);
        } else {
            const int32_t *cols[TRIE_MAX_LEVELS];
            for (int c = 0; c < nc; c++) cols[c] = rels[i]->d_cols[colord[c]];
            AMJ_TRY(build_trieN(ctx, cols, nc, rels[i]->n, &Q->triesN[i]));
            const TrieN &t = Q->triesN[i];
            g.levels = nc;
            for (int c = 0; c < nc; c++) g.data[c] = t.data[c].p;
            for (int c = 0; c + 1 < nc; c++) g.off[c] = t.off[c].p;
            g.len0 = t.len[0];
        }
        // one list per attribute at depth >= 1; a level-0 list for the first
        // attribute, and for a 1-column relation (nothing deeper implies it)
        for (int d = 0; d < nc; d++) {
            const int l = pos[rels[i]->attrs[colord[d]]];
            if (d == 0 && l != 0 && nc > 1) continue;
            GenLevel &L = Q->lv[l];
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
        for (int j = 0; j < Q->lv[l].n; j++) linked |= Q->lv[l].l[j].depth > 0;
        if (!linked)
            return fail(AMJ_EUNSUPPORTED, "LFTJ: every attribute after the first must share a relation with an earlier one");
    }
    if (Q->lv[0].n == 0) return fail(AMJ_EUNSUPPORTED, "LFTJ: no relation starts with the first attribute");
    AMJ_TRY(Q->dtries.alloc(ctx, nrels));
    AMJ_CUDA_TRY(cudaMemcpyAsync(Q->dtries.p, ht.data(), nrels * sizeof(GenTrie), cudaMemcpyHostToDevice, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return AMJ_OK;
}

// amj_lftj_execute for queries other than the triangle: a count pass, then
// with AMJ_F_MATERIALIZE a write pass into exactly allocated columns.
int lftj_generic_execute(amj_ctx *ctx, amj_rel *const *rels, int nrels, int ooc, int flags, const uint32_t *order,
                         amj_result *out) {
    if (ooc) return fail(AMJ_EUNSUPPORTED, "LFTJ: no out-of-core form beyond the triangle (the generic join is "
                                           "already memory-bounded)");
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
