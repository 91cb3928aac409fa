// ALFTJ operator host side: query discovery, trie builds, and the count /
// write / out-of-core passes of amj_lftj_execute.
//
// Reference: query_processing + LFTJ_exec (LFTJ-GPU/exec_LFTJ.cu:31-254),
// OOCWrapper::execute_with_{BFS,DFS} (LFTJ-GPU/ooc_wrapper.cuh:174-427).
// One relation is the triangle self-join (three tries share one CSR,
// exec_LFTJ.cu:96-102, 198-222); two relations are rejected
// (exec_LFTJ.cu:92-95); three relations must carry the attribute pairs
// (0,1), (1,2), (0,2).  Each trie is built with its columns in attribute
// order, as the reference orders them through a std::map (exec_LFTJ.cu:148-156).
// The relations are joined as sets, the semantics of the leapfrog triejoin:
// a repeated row counts once (the trie builds drop repeats; the reference's
// inputs are deduplicated edge lists).
#include "amj_ops.cuh"
#include "amhj_host.h"

#include <algorithm>
#include <cstring>
#include <vector>

namespace amj {
int lftj_clique4(amj_ctx *ctx, const Trie2 &T, int32_t *const *out, uint64_t out_cap, uint64_t *count,
                 uint64_t *checksum, uint64_t *written, double *kernel_ms, int sorted_out);
struct C4Matrix;
int lftj_clique4_matrix_prepare(amj_ctx *ctx, const Trie2 &T, const int32_t *inv, const uint64_t *wedge, uint64_t nv,
                                uint32_t rank_bits, C4Matrix **out);
void lftj_clique4_matrix_release(C4Matrix *m);
int lftj_clique4_matrix(amj_ctx *ctx, const Trie2 &T, const int32_t *inv, const C4Matrix *m, int32_t *const *out,
                        uint64_t out_cap, uint64_t *count, uint64_t *checksum, uint64_t *written, double *kernel_ms);
int lftj_triangle(amj_ctx *ctx, const Trie2 &R, const Trie2 &S, const Trie2 &T, int algo, int32_t *const *out,
                  uint64_t out_cap, uint64_t *count, uint64_t *checksum, uint64_t *written, int small_sum,
                  uint64_t r_lo, uint64_t r_hi, uint32_t heavy_deg, double *kernel_ms, int sorted_out,
                  const int32_t *inv, const uint64_t *wedge, uint64_t nv, uint32_t rank_bits);
int build_wedges(amj_ctx *ctx, const Trie2 &R, uint64_t nv, DBuf<uint64_t> *out);

// the generic join (lftj_generic.cu)
int lftj_generic_execute(amj_ctx *ctx, amj_rel *const *rels, int nrels, int ooc, int flags, const uint32_t *order,
                         amj_result *out);

// Trie of the self-joined edge relation: the degree-ordered copy when the
// relation is oriented and `allow` (*sorted = 1), else the relation itself.
static int build_self_trie(amj_ctx *ctx, const amj_rel *r, Trie2 *t, int *sorted, bool allow) {
    *sorted = 0;
    if (r->ncols != 2) return fail(AMJ_EUNSUPPORTED, "LFTJ: relations must have two columns");
    if (r->where == AMJ_MEM_HOST_STREAMED) return fail(AMJ_EUNSUPPORTED, "LFTJ: relations must be on the device");
    const bool swap = r->attrs[0] > r->attrs[1];
    const int32_t *c0 = r->d_cols[swap ? 1 : 0], *c1 = r->d_cols[swap ? 0 : 1];
    if (!allow) return build_trie2(ctx, c0, c1, r->n, t, true);
    DBuf<int32_t> ns, nd;
    bool oriented = false;
    AMJ_TRY(degree_ordered_copy(ctx, c0, c1, r->n, &ns, &nd, &oriented));
    if (!oriented) return build_trie2(ctx, c0, c1, r->n, t, true);
    *sorted = 1;
    return build_trie2(ctx, ns.p, nd.p, r->n, t, true);
}

// Trie of the degree-ranked copy (*inv maps ranks to vertex ids) when the
// relation is oriented, with its level-1 entries grouped by value when
// wedges is given; otherwise the trie of the relation itself, *nv = 0.
static int build_ranked_trie(amj_ctx *ctx, const amj_rel *r, Trie2 *t, DBuf<int32_t> *inv, uint64_t *nv,
                             DBuf<uint64_t> *wedges) {
    *nv = 0;
    if (r->ncols != 2) return fail(AMJ_EUNSUPPORTED, "LFTJ: relations must have two columns");
    if (r->where == AMJ_MEM_HOST_STREAMED) return fail(AMJ_EUNSUPPORTED, "LFTJ: relations must be on the device");
    const bool swap = r->attrs[0] > r->attrs[1];
    const int32_t *c0 = r->d_cols[swap ? 1 : 0], *c1 = r->d_cols[swap ? 0 : 1];
    DBuf<int32_t> ns, nd;
    bool oriented = false;
    AMJ_TRY(degree_ranked_copy(ctx, c0, c1, r->n, &ns, &nd, inv, nv, &oriented));
    if (!oriented) return build_trie2(ctx, c0, c1, r->n, t, true);
    AMJ_TRY(build_trie2_ranked(ctx, ns.p, nd.p, r->n, *nv, t));
    if (wedges) AMJ_TRY(build_wedges(ctx, *t, *nv, wedges));
    return AMJ_OK;
}
}

using namespace amj;

static int build_rel_trie(amj_ctx *ctx, const amj_rel *r, Trie2 *t) {
    if (r->ncols != 2) return fail(AMJ_EUNSUPPORTED, "LFTJ: relations must have two columns");
    if (r->where == AMJ_MEM_HOST_STREAMED) return fail(AMJ_EUNSUPPORTED, "LFTJ: relations must be on the device");
    const bool swap = r->attrs[0] > r->attrs[1];
    return build_trie2(ctx, r->d_cols[swap ? 1 : 0], r->d_cols[swap ? 0 : 1], r->n, t, true);
}

// The 4-clique over one edge relation (AMJ_F_CLIQUE4): a count pass, then
// with AMJ_F_MATERIALIZE a write pass into exactly allocated columns.  With
// matrices_only the query runs only where the triangle matrices apply;
// otherwise *used is false and nothing is reported.
static int lftj_clique4_execute(amj_ctx *ctx, amj_rel *const *rels, int nrels, int algo, int ooc, int flags,
                                amj_result *out, bool matrices_only = false, bool *used = nullptr) {
    if (nrels != 1) return fail(AMJ_EUNSUPPORTED, "LFTJ 4-clique: one edge relation");
    if (algo != AMJ_LFTJ_DFS) return fail(AMJ_EUNSUPPORTED, "LFTJ 4-clique: DFS only");
    if (used) *used = false;
    result_init(out, 4);
    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1], e2 = ctx->ev[2];
    AMJ_CUDA_TRY(cudaEventRecord(e0, ctx->stream));
    Trie2 t;
    int sorted_out = 0;
    // an oriented relation with out-degrees up to 1024 in degree order: the
    // triangle matrices of its degree-ranked copy; otherwise the 4-clique
    // kernel over the degree-ordered copy (or the relation as given)
    DBuf<int32_t> inv;
    uint64_t nv = 0;
    struct MatGuard {
        C4Matrix *m = nullptr;
        ~MatGuard() { lftj_clique4_matrix_release(m); }
    } mat;
    if ((flags & AMJ_F_KEEP_ORDER) == 0 && (flags & AMJ_F_CLIQUE4_LISTS)) {
        AMJ_TRY(build_self_trie(ctx, rels[0], &t, &sorted_out, true));
    } else if ((flags & AMJ_F_KEEP_ORDER) == 0) {
        DBuf<uint64_t> wedges;
        AMJ_TRY(build_ranked_trie(ctx, rels[0], &t, &inv, &nv, &wedges));
        // the hash join's bag semantics: only a relation that is oriented
        // and has no repeated rows (the trie dropped none) joins as a set
        if (matrices_only && (!nv || t.len1 != rels[0]->n)) return AMJ_OK;
        if (nv) {
            AMJ_TRY(lftj_clique4_matrix_prepare(ctx, t, inv.p, wedges.p, nv, ctx->opts.lftj_rank_bits, &mat.m));
            if (!mat.m && matrices_only) return AMJ_OK;
            if (!mat.m) {
                t = Trie2();
                inv.release();
                AMJ_TRY(build_self_trie(ctx, rels[0], &t, &sorted_out, true));
            }
        }
    } else {
        AMJ_TRY(build_self_trie(ctx, rels[0], &t, &sorted_out, false));
    }
    if (used) *used = true;
    AMJ_CUDA_TRY(cudaEventRecord(e1, ctx->stream));
    uint64_t c = 0, h = 0;
    if (mat.m)
        AMJ_TRY(lftj_clique4_matrix(ctx, t, inv.p, mat.m, nullptr, 0, &c, &h, nullptr, &out->kernel_ms[0]));
    else
        AMJ_TRY(lftj_clique4(ctx, t, nullptr, 0, &c, &h, nullptr, &out->kernel_ms[0], sorted_out));
    out->count = c;
    out->checksum = h;
    const bool materialize = (flags & AMJ_F_MATERIALIZE) != 0;
    if (materialize) {
        int32_t *cols[4] = {nullptr, nullptr, nullptr, nullptr};
        int rc = AMJ_OK;
        for (int a = 0; a < 4 && rc == AMJ_OK; a++) rc = dev_alloc(ctx, (void **)&cols[a], (c ? c : 1) * 4);
        uint64_t c2 = 0, h2 = 0, w = 0;
        if (rc == AMJ_OK)
            rc = mat.m ? lftj_clique4_matrix(ctx, t, inv.p, mat.m, cols, c, &c2, &h2, &w, &out->kernel_ms[1])
                       : lftj_clique4(ctx, t, cols, c, &c2, &h2, &w, &out->kernel_ms[1], sorted_out);
        if (rc == AMJ_OK && (c2 != c || h2 != h || w != c))
            rc = fail(AMJ_ECUDA, "LFTJ 4-clique: write pass disagrees with count pass");
        if (rc != AMJ_OK) {
            for (int a = 0; a < 4; a++) dev_free(ctx, cols[a]);
            return rc;
        }
        auto *o = new ResultOwner();
        o->ctx = ctx;
        out->priv = o;
        out->rows = c;
        for (int a = 0; a < 4; a++) out->cols[a] = cols[a];
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

// AMHJ FOUR over one oriented edge relation (exec_AMHJ.cu:53-69): the last
// three levels of the hash-join plan, R(0,3), R(1,3), R(2,3), look up the
// fourth vertex by the pair keys of an edge and a triangle.  On the
// degree-ranked copy those lookups are one AND of two rows of the triangle
// matrix of the first vertex (lftj_clique4.cu); where the matrices apply
// (out-degrees up to 1024 and memory for them) the query runs that way and
// *used is true.
int amj::amhj_four_by_matrices(amj_ctx *ctx, amj_rel *rel, int flags, amj_result *out, bool *used) {
    amj_rel *rels[1] = {rel};
    return lftj_clique4_execute(ctx, rels, 1, AMJ_LFTJ_DFS, 0, flags & ~(AMJ_F_CLIQUE4_LISTS | AMJ_F_KEEP_ORDER), out,
                                true, used);
}

static int triangle_run(amj_ctx *ctx, const Trie2 &R_, const Trie2 &S_, const Trie2 &T_, int algo, int ws,
                        int flags, int sorted_out, const int32_t *rank_inv, const uint64_t *wedge, uint64_t nv,
                        amj_result *out);

// AMHJ TRI over one oriented edge relation (exec_AMHJ.cu:32-49): the levels
// R(0,2) keyed on a and the pair-key filter R(1,2) become, on the
// degree-ranked copy, the suffix of a's child list after b tested against a
// bitmap of b's children (the wedge kernel, lftj.cu).  Taken where the
// relation is oriented and has no repeated rows (the hash join counts
// repeats, the trie joins sets); otherwise *used is false.
int amj::amhj_tri_by_wedges(amj_ctx *ctx, amj_rel *rel, int flags, amj_result *out, bool *used) {
    *used = false;
    result_init(out, 3);
    AMJ_CUDA_TRY(cudaEventRecord(ctx->ev[0], ctx->stream));
    Trie2 t;
    DBuf<int32_t> inv;
    DBuf<uint64_t> wedges;
    uint64_t nv = 0;
    AMJ_TRY(build_ranked_trie(ctx, rel, &t, &inv, &nv, &wedges));
    if (!nv || t.len1 != rel->n) return AMJ_OK;
    *used = true;
    return triangle_run(ctx, t, t, t, AMJ_LFTJ_DFS, 1, flags, 1, inv.p, wedges.p, nv, out);
}

// The self-joined edge relation as the relations of the triangle (TRI
// pattern) or 4-clique (FOUR pattern), for the generic join in a given
// attribute order: views of the same device columns, none owning them.
static int self_join_views(const amj_rel *r, bool clique4, amj_rel *views, amj_rel **ptrs, int *n) {
    if (r->ncols != 2) return fail(AMJ_EUNSUPPORTED, "LFTJ: relations must have two columns");
    static const uint32_t tri[3][2] = {{0, 1}, {1, 2}, {0, 2}};
    static const uint32_t four[6][2] = {{0, 1}, {1, 2}, {2, 3}, {0, 3}, {0, 2}, {1, 3}};
    const bool swap = r->attrs[0] > r->attrs[1];
    *n = clique4 ? 6 : 3;
    for (int i = 0; i < *n; i++) {
        views[i] = amj_rel();
        views[i].ctx = r->ctx;
        views[i].n = r->n;
        views[i].ncols = 2;
        views[i].where = r->where;
        views[i].owned = false;
        views[i].d_cols[0] = r->d_cols[swap ? 1 : 0];
        views[i].d_cols[1] = r->d_cols[swap ? 0 : 1];
        views[i].h_cols[0] = r->h_cols[swap ? 1 : 0];
        views[i].h_cols[1] = r->h_cols[swap ? 0 : 1];
        views[i].attrs[0] = clique4 ? four[i][0] : tri[i][0];
        views[i].attrs[1] = clique4 ? four[i][1] : tri[i][1];
        ptrs[i] = &views[i];
    }
    return AMJ_OK;
}

static bool identity_order(const uint32_t *order, int k) {
    if (!order) return true;
    for (int i = 0; i < k; i++)
        if (order[i] != (uint32_t)i) return false;
    return true;
}

static int lftj_execute_impl(amj_ctx *ctx, amj_rel *const *rels, int nrels, int algo, int ooc, int ws, int flags,
                             const uint32_t *order, int norder, amj_result *out);

extern "C" int amj_lftj_execute(amj_ctx *ctx, amj_rel *const *rels, int nrels, int algo, int ooc, int ws, int flags,
                                amj_result *out) {
    return lftj_execute_impl(ctx, rels, nrels, algo, ooc, ws, flags, nullptr, 0, out);
}

extern "C" int amj_lftj_execute_ordered(amj_ctx *ctx, amj_rel *const *rels, int nrels, int algo, int ooc, int ws,
                                        int flags, const uint32_t *attr_order, int k, amj_result *out) {
    if (attr_order && (k <= 0 || k > AMJ_MAX_ATTRS)) return fail(AMJ_EINVAL, "lftj_execute: bad attribute order length");
    return lftj_execute_impl(ctx, rels, nrels, algo, ooc, ws, flags, attr_order, attr_order ? k : 0, out);
}

// The triangle over tries R(0,1), S(1,2), T(0,2) built since ctx->ev[0]
// was recorded: a count pass, with AMJ_F_MATERIALIZE a write pass into
// exactly allocated columns, and the result's timings.
static int triangle_run(amj_ctx *ctx, const Trie2 &R_, const Trie2 &S_, const Trie2 &T_, int algo, int ws,
                        int flags, int sorted_out, const int32_t *rank_inv, const uint64_t *wedge, uint64_t nv,
                        amj_result *out) {
    const Trie2 *R = &R_, *S = &S_, *T = &T_;
    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1], e2 = ctx->ev[2];
    AMJ_CUDA_TRY(cudaEventRecord(e1, ctx->stream));

    // ws=0: every (a,b) pair intersected by its own lane; ws=1: long pairs
    // shared by the whole warp
    const int small_sum = ws ? 48 : 0x7fffffff;
    // ws=1 also hands vertices with many children to the block-wide bitmap kernel
    const uint32_t heavy_deg = ws ? (ctx->opts.lftj_heavy_degree ? ctx->opts.lftj_heavy_degree : 32u) : 0u;
    const bool materialize = (flags & AMJ_F_MATERIALIZE) != 0;
    const uint64_t nr = R->len1;
    uint64_t c = 0, h = 0, w = 0;
    int rc = lftj_triangle(ctx, *R, *S, *T, algo, nullptr, 0, &c, &h, nullptr, small_sum, 0, nr, heavy_deg,
                           out->kernel_ms, sorted_out, rank_inv, wedge, nv, ctx->opts.lftj_rank_bits);
    if (rc != AMJ_OK) return rc;
    int32_t *dcols[3] = {nullptr, nullptr, nullptr};
    if (materialize) {
        for (int a = 0; a < 3 && rc == AMJ_OK; a++) rc = dev_alloc(ctx, (void **)&dcols[a], (c ? c : 1) * 4);
        uint64_t c2 = 0, h2 = 0;
        if (rc == AMJ_OK)
            rc = lftj_triangle(ctx, *R, *S, *T, algo, dcols, c, &c2, &h2, &w, small_sum, 0, nr, heavy_deg,
                               out->kernel_ms + 2, sorted_out, rank_inv, wedge, nv, ctx->opts.lftj_rank_bits);
        if (rc == AMJ_OK && (c2 != c || h2 != h || w != c))
            rc = fail(AMJ_ECUDA, "LFTJ: write pass disagrees with count pass");
        if (rc != AMJ_OK) {
            for (int a = 0; a < 3; a++) dev_free(ctx, dcols[a]);
            return rc;
        }
    }
    out->count = c;
    out->checksum = h;
    out->stats[7] = 1;
    if (materialize) {
        auto *o = new ResultOwner();
        o->ctx = ctx;
        out->priv = o;
        out->rows = c;
        for (int a = 0; a < 3; a++) out->cols[a] = dcols[a];
    }
    AMJ_CUDA_TRY(cudaEventRecord(e2, ctx->stream));
    AMJ_CUDA_TRY(cudaEventSynchronize(e2));
    out->build_ms = event_ms(e0, e1);
    out->probe_ms = event_ms(e1, e2);
    out->total_ms = event_ms(e0, e2);
    if (materialize) {
        rc = finish_result_columns(ctx, out, flags);
        if (rc != AMJ_OK) {
            amj_result_release(out);
            return rc;
        }
    }
    return AMJ_OK;
}

static int lftj_execute_impl(amj_ctx *ctx, amj_rel *const *rels, int nrels, int algo, int ooc, int ws, int flags,
                             const uint32_t *order, int norder, amj_result *out) {
    if (!ctx || !out || !rels || nrels <= 0) return fail(AMJ_EINVAL, "lftj_execute: bad arguments");
    if (algo != AMJ_LFTJ_BFS && algo != AMJ_LFTJ_DFS) return fail(AMJ_EINVAL, "lftj_execute: algo must be 0 (BFS) or 1 (DFS)");
    if (nrels == 2) return fail(AMJ_EINVAL, "lftj_execute: wrong number of datasets: 2");
    for (int i = 0; i < nrels; i++)
        if (!rels[i]) return fail(AMJ_EINVAL, "lftj_execute: null relation");
    if (nrels > 16) return fail(AMJ_EUNSUPPORTED, "lftj_execute: at most 16 relations");
    AMJ_CUDA_TRY(cudaSetDevice(ctx->device));
    if (ooc || !identity_order(order, norder)) {
        // out-of-core (value-range trie slices under a memory budget), or a
        // binding order other than the identity: the generic join, which
        // reports every tuple in attribute-id order
        if (nrels == 1) {
            amj_rel views[6];
            amj_rel *ptrs[6];
            int nv = 0;
            AMJ_TRY(self_join_views(rels[0], (flags & AMJ_F_CLIQUE4) != 0, views, ptrs, &nv));
            return lftj_generic_execute(ctx, ptrs, nv, ooc, flags, order, out);
        }
        if (flags & AMJ_F_CLIQUE4) return fail(AMJ_EUNSUPPORTED, "LFTJ 4-clique: one edge relation");
        return lftj_generic_execute(ctx, rels, nrels, ooc, flags, order, out);
    }
    if (flags & AMJ_F_CLIQUE4) return lftj_clique4_execute(ctx, rels, nrels, algo, ooc, flags, out);
    if (nrels >= 3) {
        // the triangle pattern (0,1), (1,2), (0,2) keeps its own kernels; any
        // other query goes to the generic join (the reference stops at 3 tables)
        bool tri = nrels == 3;
        uint32_t pairs = 0;
        for (int i = 0; i < nrels && tri; i++) {
            if (rels[i]->ncols != 2) {
                tri = false;
                break;
            }
            const uint32_t lo = std::min(rels[i]->attrs[0], rels[i]->attrs[1]);
            const uint32_t hi = std::max(rels[i]->attrs[0], rels[i]->attrs[1]);
            const uint32_t bit = (lo == 0 && hi == 1) ? 1u : (lo == 1 && hi == 2) ? 2u : (lo == 0 && hi == 2) ? 4u : 0u;
            if (!bit || (pairs & bit)) tri = false;
            pairs |= bit;
        }
        if (!tri) return lftj_generic_execute(ctx, rels, nrels, ooc, flags, nullptr, out);
    }
    result_init(out, 3);
    AMJ_CUDA_TRY(cudaEventRecord(ctx->ev[0], ctx->stream));

    Trie2 tries[3];
    const Trie2 *R = nullptr, *S = nullptr, *T = nullptr;
    int sorted_out = 0;
    DBuf<int32_t> inv;   // ranks to vertex ids, for a degree-ranked trie
    DBuf<uint64_t> wedges;   // its level-1 entries grouped by b
    uint64_t nv = 0;
    if (nrels == 1) {
        // BFS and the DFS wedge kernel (ws=1) join the degree-ranked copy:
        // hubs keep short child lists
        bool deg_order = algo == AMJ_LFTJ_BFS || ws;
        if (flags & AMJ_F_DEGREE_ORDER) deg_order = true;
        if (flags & AMJ_F_KEEP_ORDER) deg_order = false;
        if (deg_order && (algo == AMJ_LFTJ_BFS || ws)) {
            // the degree-ranked copy: the wedge kernel (DFS) or wedge candidates (BFS)
            AMJ_TRY(build_ranked_trie(ctx, rels[0], &tries[0], &inv, &nv,
                                      algo == AMJ_LFTJ_DFS ? &wedges : nullptr));
            sorted_out = nv ? 1 : 0;
        } else {
            AMJ_TRY(build_self_trie(ctx, rels[0], &tries[0], &sorted_out, deg_order));
        }
        R = S = T = &tries[0];
    } else {
        for (int i = 0; i < 3; i++) {
            if (rels[i]->ncols != 2) return fail(AMJ_EUNSUPPORTED, "LFTJ: relations must have two columns");
            const uint32_t lo = std::min(rels[i]->attrs[0], rels[i]->attrs[1]);
            const uint32_t hi = std::max(rels[i]->attrs[0], rels[i]->attrs[1]);
            const Trie2 **slot = (lo == 0 && hi == 1) ? &R : (lo == 1 && hi == 2) ? &S : (lo == 0 && hi == 2) ? &T : nullptr;
            if (!slot || *slot)
                return fail(AMJ_EUNSUPPORTED, "LFTJ: three relations must carry attributes (0,1), (1,2) and (0,2)");
            AMJ_TRY(build_rel_trie(ctx, rels[i], &tries[i]));
            *slot = &tries[i];
        }
    }
    return triangle_run(ctx, *R, *S, *T, algo, ws, flags, sorted_out, nv ? inv.p : nullptr, wedges.p, nv, out);
}
