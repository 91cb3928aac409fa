// ALFTJ for any connected query over 2-column relations, up to AMJ_MAX_ATTRS
// attributes in identity order (the reference's attribute order,
// LFTJ-GPU/exec_LFTJ.cu:231; its LFTJ stops at 3 attributes and 3 tables,
// LFTJ-GPU/config.h:16-17).
//
// Every relation R(x, y), x < y, becomes a trie keyed on x.  Attribute 0
// ranges over the intersection of the level-0 arrays of the relations keyed
// on it; attribute l >= 1 over the intersection of the child lists
// R(v_x) of the relations closing it (those with y = l).  The join is
// level-synchronous (the leapfrog of LFTJ_BFS, LFTJ-GPU/LFTJ_BFS.cuh:143-500,
// generalised): per level one count kernel takes, for every partial tuple,
// its shortest list; the candidates of all tuples form one space, which is
// cut into pieces of bounded size; per piece an expand kernel tests each
// candidate against the tuple's other lists (binary search) and either
// counts and hashes finished tuples (last attribute) or keeps survivors,
// which a scan compacts into the next level's tuples.  Memory stays bounded
// by the piece size whatever the intermediate results.
// Lists are strictly increasing (relations without duplicate tuples).
#include "lftj_common.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace amj {

constexpr int GEN_MAX_LISTS = 8;                 // relations closing one attribute
constexpr uint64_t GEN_PIECE = 1ull << 26;       // candidates per expand launch

// the lists that constrain one attribute
struct GenLevel {
    int n;
    TrieRef t[GEN_MAX_LISTS];
    int8_t parent[GEN_MAX_LISTS];                // attribute whose value keys the list; -1: level 0
};

struct GenArgs {
    GenLevel L;
    int level;                                   // attribute being bound
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
};

// range [s, e) of list i for tuple t, in the list's value array *base
__device__ __forceinline__ void gen_range(const GenLevel &L, int i, const int32_t *const *cols, uint64_t t,
                                          const int32_t *&base, uint64_t &s, uint64_t &e) {
    if (L.parent[i] < 0) {
        base = L.t[i].data0;
        s = 0;
        e = L.t[i].len0;
    } else {
        base = L.t[i].data1;
        child_range(L.t[i], cols[L.parent[i]][t], s, e);
    }
}

__global__ void gen_count_kernel(const __grid_constant__ GenArgs A, unsigned long long *cnt) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < A.F; t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t best = ~0ull, bs = 0;
        int bi = 0;
        for (int i = 0; i < A.L.n; i++) {
            const int32_t *base;
            uint64_t s, e;
            gen_range(A.L, i, A.cols, t, base, s, e);
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

// first index in [s, e) of base with value >= v
__device__ __forceinline__ uint64_t gen_lower(const int32_t *base, uint64_t s, uint64_t e, int32_t v) {
    while (s < e) {
        const uint64_t m = (s + e) >> 1;
        if (base[m] < v) s = m + 1;
        else e = m;
    }
    return s;
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
        gen_range(A.L, si, A.cols, t, sbase, ss, se);
        const int32_t c = sbase[A.sbeg[t] + (g - A.offs[t])];
        bool keep = true;
        for (int i = 0; i < A.L.n && keep; i++) {
            if (i == si) continue;
            const int32_t *base;
            uint64_t s, e;
            gen_range(A.L, i, A.cols, t, base, s, e);
            const uint64_t p = gen_lower(base, s, e, c);
            keep = p < e && base[p] == c;
        }
        if (!A.last) {
            A.keep[g - A.g0] = keep ? 1u : 0u;
            A.val[g - A.g0] = c;
            continue;
        }
        if (!keep) continue;
        uint64_t h = AMJ_CHECKSUM_SEED;
        for (int a = 0; a < A.level; a++) h = amj_hash_step(h, A.cols[a][t]);
        h = amj_hash_step(h, c);
        cnt++;
        chk += h;
        if (WRITE) {
            const unsigned long long p = atomicAdd(A.out_cursor, 1ull);
            if (p < A.out_cap) {
                for (int a = 0; a < A.level; a++) A.out[a][p] = A.cols[a][t];
                A.out[A.level][p] = c;
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
    std::vector<Trie2> tries;
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
    A.level = level;
    A.last = level == Q.k - 1;
    A.k = Q.k;
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

// Compile a query of 2-column relations: attributes 0..k-1, every attribute
// but the first closed by at least one relation with an earlier attribute.
int lftj_generic_compile(amj_ctx *ctx, amj_rel *const *rels, int nrels, GenQuery *Q) {
    uint32_t seen = 0;
    for (int i = 0; i < nrels; i++) {
        if (rels[i]->ncols != 2) return fail(AMJ_EUNSUPPORTED, "LFTJ: relations must have two columns");
        if (rels[i]->where == AMJ_MEM_HOST_STREAMED)
            return fail(AMJ_EUNSUPPORTED, "LFTJ: relations must be on the device");
        if (rels[i]->attrs[0] == rels[i]->attrs[1]) return fail(AMJ_EINVAL, "LFTJ: a relation repeats an attribute");
        seen |= (1u << rels[i]->attrs[0]) | (1u << rels[i]->attrs[1]);
    }
    int k = 0;
    while (k < 32 && ((seen >> k) & 1)) k++;
    if (seen != ((1u << k) - 1) || k > AMJ_MAX_ATTRS)
        return fail(AMJ_EINVAL, "LFTJ: the relations' attributes must be exactly 0..k-1 with k <= 8");
    Q->k = k;
    Q->tries.resize(nrels);
    for (int l = 0; l < k; l++) Q->lv[l].n = 0;
    for (int i = 0; i < nrels; i++) {
        const bool swap = rels[i]->attrs[0] > rels[i]->attrs[1];
        const int x = (int)(swap ? rels[i]->attrs[1] : rels[i]->attrs[0]);
        const int y = (int)(swap ? rels[i]->attrs[0] : rels[i]->attrs[1]);
        AMJ_TRY(build_trie2(ctx, rels[i]->d_cols[swap ? 1 : 0], rels[i]->d_cols[swap ? 0 : 1], rels[i]->n,
                            &Q->tries[i], true));
        const TrieRef tr = trie_ref(Q->tries[i]);
        if (Q->lv[y].n >= GEN_MAX_LISTS) return fail(AMJ_EUNSUPPORTED, "LFTJ: more than 8 relations close one attribute");
        Q->lv[y].t[Q->lv[y].n] = tr;
        Q->lv[y].parent[Q->lv[y].n] = (int8_t)x;
        Q->lv[y].n++;
        if (x == 0) {
            if (Q->lv[0].n >= GEN_MAX_LISTS) return fail(AMJ_EUNSUPPORTED, "LFTJ: more than 8 relations on attribute 0");
            Q->lv[0].t[Q->lv[0].n] = tr;
            Q->lv[0].parent[Q->lv[0].n] = -1;
            Q->lv[0].n++;
        }
    }
    for (int l = 1; l < k; l++)
        if (Q->lv[l].n == 0)
            return fail(AMJ_EUNSUPPORTED, "LFTJ: every attribute after the first must share a relation with an earlier one");
    return AMJ_OK;
}

// amj_lftj_execute for queries other than the triangle: a count pass, then
// with AMJ_F_MATERIALIZE a write pass into exactly allocated columns.
int lftj_generic_execute(amj_ctx *ctx, amj_rel *const *rels, int nrels, int ooc, int flags, amj_result *out) {
    if (ooc) return fail(AMJ_EUNSUPPORTED, "LFTJ: no out-of-core form beyond the triangle (the generic join is "
                                           "already memory-bounded)");
    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1], e2 = ctx->ev[2];
    AMJ_CUDA_TRY(cudaEventRecord(e0, ctx->stream));
    GenQuery Q;
    AMJ_TRY(lftj_generic_compile(ctx, rels, nrels, &Q));
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
