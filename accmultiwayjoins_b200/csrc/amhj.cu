// AMHJ operator host side: query compilation, index builds, and the count /
// write / direct-output / work-sharing / out-of-core passes.
//
// Reference entry: test_general + OOC::execute (MHJ-GPU/exec_AMHJ.cu:10-213,
// MHJ-GPU/ooc.cuh:77-307) dispatching AMHJ / AMHJ_WS / AMHJ_DRO / AMHJ_WS_DRO /
// AMHJ_FIB (exec_AMHJ.cu:163-198).
//
// Query compilation follows exec_AMHJ.cu:70-89 (NORMAL) and the hard-coded
// TRI / FOUR attribute patterns (exec_AMHJ.cu:32-69, 126-138): an attribute
// already bound by an earlier relation is compared, a new one is bound.  All
// bound attributes are compared (the reference's single_join_key=false
// semantics, common_kernels.cuh:41-53).  Two choices differ from the
// reference and leave the result bag unchanged:
//  - a build relation whose columns are all bound (a pure filter, e.g. C(0,2)
//    of the triangle) is indexed on the pair of its columns, so its lookup is
//    one bucket instead of a scan of every row sharing the first value;
//  - such filters move to the earliest level at which their attributes are
//    bound (AMJ_F_NO_REORDER keeps the query order).
#include "amhj_host.h"
#include "amhj_star.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

namespace amj {

struct RelAttrs {
    const amj_rel *rel;
    int ncols;
    int attr[AMJ_MAX_COLS];
};

int compile_plan(int query_type, amj_rel *const *rels, int nrels, int flags, HostPlan *hp) {
    std::vector<RelAttrs> tabs;
    if (query_type == AMJ_QUERY_NORMAL) {
        if (nrels < 1) return fail(AMJ_EINVAL, "AMHJ: no relations");
        if (nrels - 1 > AMJ_MAX_BUILD_TABLES) return fail(AMJ_EUNSUPPORTED, "AMHJ: more than 6 build relations");
        for (int i = 0; i < nrels; i++) {
            RelAttrs t{rels[i], rels[i]->ncols, {}};
            for (int c = 0; c < t.ncols; c++) t.attr[c] = (int)rels[i]->attrs[c];
            tabs.push_back(t);
        }
    } else if (query_type == AMJ_QUERY_TRI || query_type == AMJ_QUERY_FOUR) {
        if (nrels != 1 || rels[0]->ncols != 2)
            return fail(AMJ_EINVAL, "AMHJ TRI/FOUR: expected one 2-column edge relation");
        // A(0,1),B(1,2),C(0,2)  /  A(0,1),B(1,2),C(2,3),D(0,3),E(0,2),F(1,3)
        static const int tri[3][2] = {{0, 1}, {1, 2}, {0, 2}};
        static const int four[6][2] = {{0, 1}, {1, 2}, {2, 3}, {0, 3}, {0, 2}, {1, 3}};
        const int nt = query_type == AMJ_QUERY_TRI ? 3 : 6;
        for (int i = 0; i < nt; i++) {
            RelAttrs t{rels[0], 2, {}};
            t.attr[0] = query_type == AMJ_QUERY_TRI ? tri[i][0] : four[i][0];
            t.attr[1] = query_type == AMJ_QUERY_TRI ? tri[i][1] : four[i][1];
            tabs.push_back(t);
        }
    } else {
        return fail(AMJ_EINVAL, "AMHJ: unknown query type");
    }
    // attributes must be exactly 0..k-1
    uint32_t seen = 0;
    for (auto &t : tabs)
        for (int c = 0; c < t.ncols; c++) seen |= 1u << t.attr[c];
    int k = 0;
    while (k < 32 && ((seen >> k) & 1)) k++;
    if (seen != ((1u << k) - 1) || k > AMJ_MAX_ATTRS)
        return fail(AMJ_EINVAL, "AMHJ: the relations' attributes must be exactly 0..k-1 with k <= 8");
    hp->k = k;
    hp->probe = tabs[0].rel;
    for (int c = 0; c < tabs[0].ncols; c++) hp->probe_attr[c] = tabs[0].attr[c];
    uint32_t bound = 0;
    for (int c = 0; c < tabs[0].ncols; c++) bound |= 1u << tabs[0].attr[c];
    // the build relations not placed yet, in query order
    std::vector<size_t> rem;
    for (size_t i = 1; i < tabs.size(); i++) rem.push_back(i);
    int L = 0;
    while (!rem.empty()) {
        size_t pick = 0;
        if (!(flags & AMJ_F_NO_REORDER)) {
            for (size_t i = 0; i < rem.size(); i++) {
                const RelAttrs &r = tabs[rem[i]];
                bool all = true;
                for (int c = 0; c < r.ncols; c++) all &= ((bound >> r.attr[c]) & 1) != 0;
                if (all) {
                    pick = i;
                    break;
                }
            }
        }
        const RelAttrs t = tabs[rem[pick]];
        for (size_t i = pick + 1; i < rem.size(); i++) rem[i - 1] = rem[i];
        rem.pop_back();
        if (t.ncols > 4) return fail(AMJ_EUNSUPPORTED, "AMHJ: build relations have at most 4 columns");
        int kc = -1;   // key column: the first column whose attribute is bound
        for (int c = 0; c < t.ncols && kc < 0; c++)
            if ((bound >> t.attr[c]) & 1) kc = c;
        if (kc < 0) return fail(AMJ_EUNSUPPORTED, "AMHJ: a build relation shares no attribute with the relations before it");
        LevelSpec &ls = hp->lv[L];
        ls.rel = t.rel;
        ls.ncols = t.ncols;
        int w = 0;
        ls.src_col[w] = kc;
        ls.attr[w++] = t.attr[kc];
        for (int c = 0; c < t.ncols; c++)
            if (c != kc) {
                ls.src_col[w] = c;
                ls.attr[w++] = t.attr[c];
            }
        ls.cmp_mask = ls.bind_mask = 0;
        for (int c = 0; c < t.ncols; c++) {
            if ((bound >> ls.attr[c]) & 1) ls.cmp_mask |= 1u << c;
            else ls.bind_mask |= 1u << c;
        }
        ls.key_mode = (t.ncols == 2 && ls.cmp_mask == 3u) ? KEY_PAIR : KEY_SINGLE;
        for (int c = 0; c < t.ncols; c++) bound |= 1u << ls.attr[c];
        L++;
    }
    hp->L = L;
    return AMJ_OK;
}


struct ExecScratch {
    std::map<IndexKey, HashIndex> indexes;
    DBuf<ProbeState> st;
    DBuf<Task> tasks;
    DBuf<unsigned int> ready;
    DBuf<Breakpoint> units;
    // frequent-item buffer
    DBuf<int32_t> fib_keys;
    DBuf<uint32_t> fib_idx;
    DBuf<unsigned long long> fib_off;
    DBuf<int32_t> fib_cols[AMJ_MAX_ATTRS];
};

double event_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0.0;
    }
    return (double)ms;
}

template <int MODE, bool WS, bool WT>
static int launch_probe_t(amj_ctx *ctx, const ProbeLaunch &PL, size_t smem) {
    auto kern = amhj_probe_kernel<MODE, WS, WT>;
    AMJ_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    AMJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, PROBE_THREADS, smem));
    if (per_sm < 1) return fail(AMJ_EUNSUPPORTED, "AMHJ: probe frontier does not fit in shared memory");
    uint64_t grid = (uint64_t)ctx->num_sms * per_sm;
    if (ctx->opts.max_blocks && grid > ctx->opts.max_blocks) grid = ctx->opts.max_blocks;
    const uint64_t need = (PL.batch_count + PROBE_WARPS - 1) / PROBE_WARPS;
    if (!WS && MODE != PM_RESIDUAL && need < grid) grid = need ? need : 1;
    if (MODE == PM_RESIDUAL) {
        const uint64_t rneed = (PL.batch_count + PROBE_WARPS - 1) / PROBE_WARPS;
        if (rneed < grid) grid = rneed ? rneed : 1;
    }
    if (WS) {
        // every warp starts counted as busy
        const unsigned int warps = (unsigned int)(grid * PROBE_WARPS);
        AMJ_CUDA_TRY(cudaMemcpyAsync(&PL.st->busy, &warps, sizeof(warps), cudaMemcpyHostToDevice, ctx->stream));
    }
    note_launch(ctx);
    kern<<<(unsigned)grid, PROBE_THREADS, smem, ctx->stream>>>(PL);
    AMJ_CUDA_TRY(cudaGetLastError());
    return AMJ_OK;
}

static int launch_probe_raw(amj_ctx *ctx, const ProbeLaunch &PL, int mode, bool ws) {
    const size_t smem = (size_t)PROBE_WARPS * PL.P.warp_bytes;
    const bool wt = PL.P.has_inl != 0;
#define AMJ_LAUNCH(M)                                                                              \
    return ws ? (wt ? launch_probe_t<M, true, true>(ctx, PL, smem) : launch_probe_t<M, true, false>(ctx, PL, smem)) \
              : (wt ? launch_probe_t<M, false, true>(ctx, PL, smem) : launch_probe_t<M, false, false>(ctx, PL, smem))
    if (mode == PM_COUNT) AMJ_LAUNCH(PM_COUNT);
    if (mode == PM_WRITE) AMJ_LAUNCH(PM_WRITE);
    AMJ_LAUNCH(PM_RESIDUAL);
#undef AMJ_LAUNCH
}

// probe launch bracketed by the context's kernel-timing events
static int launch_probe(amj_ctx *ctx, const ProbeLaunch &PL, int mode, bool ws) {
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[0], ctx->stream));
    AMJ_TRY(launch_probe_raw(ctx, PL, mode, ws));
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[1], ctx->stream));
    return AMJ_OK;
}

static int reset_state(amj_ctx *ctx, ProbeState *st, unsigned int *ready, uint32_t task_cap) {
    AMJ_CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(ProbeState), ctx->stream));
    if (ready) AMJ_CUDA_TRY(cudaMemsetAsync(ready, 0, (size_t)task_cap * sizeof(unsigned int), ctx->stream));
    return AMJ_OK;
}

// read the probe state back after the last launch; adds that launch's
// kernel time to *kslot when given
static int read_state(amj_ctx *ctx, const ProbeState *d, ProbeState *h, const char *what, double *kslot = nullptr) {
    AMJ_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(ProbeState), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_TRY(status_check(ctx, what));
    if (kslot) *kslot += event_ms(ctx->kev[0], ctx->kev[1]);
    return AMJ_OK;
}

static int alloc_cols(amj_ctx *ctx, int k, uint64_t rows, int32_t **cols) {
    for (int a = 0; a < k; a++) {
        int rc = dev_alloc(ctx, (void **)&cols[a], (rows ? rows : 1) * sizeof(int32_t));
        if (rc != AMJ_OK) {
            for (int b = 0; b < a; b++) dev_free(ctx, cols[b]);
            return rc;
        }
    }
    return AMJ_OK;
}

int finish_result_columns(amj_ctx *ctx, amj_result *res, int flags) {
    if (!(flags & AMJ_F_HOST_RESULT) || res->on_host) return AMJ_OK;
    int32_t *host[AMJ_MAX_ATTRS] = {};
    for (int a = 0; a < res->num_attrs; a++) {
        if (!res->cols[a]) continue;
        if (cudaMallocHost((void **)&host[a], (res->rows ? res->rows : 1) * sizeof(int32_t)) != cudaSuccess) {
            (void)cudaGetLastError();
            for (int b = 0; b < a; b++) cudaFreeHost(host[b]);
            return fail(AMJ_ENOMEM, "result: pinned host allocation failed");
        }
        if (res->rows)
            AMJ_CUDA_TRY(cudaMemcpyAsync(host[a], res->cols[a], res->rows * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                         ctx->stream));
    }
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int a = 0; a < res->num_attrs; a++) {
        if (!res->cols[a]) continue;
        dev_free(ctx, res->cols[a]);
        res->cols[a] = host[a];
    }
    res->on_host = 1;
    return AMJ_OK;
}

// Everything of one execute call except the index builds: the passes over
// probe rows [row_lo, row_hi).  Accumulates into *res (count, checksum,
// stats); with materialise, appends rows to `out` (device columns with
// `out_cap` rows from `out_base`) and reports rows written.
struct PassResult {
    uint64_t count = 0, checksum = 0, rows = 0;
    int32_t *cols[AMJ_MAX_ATTRS] = {};
};

static int run_passes(amj_ctx *ctx, ProbeLaunch &PL, ExecScratch &X, bool ws, bool dro, bool materialize,
                      uint64_t row_lo, uint64_t row_hi, PassResult *pr, amj_result *res, bool allow_flat = true);

// Count mode of a star or canonical chain plan (amhj_star.cuh): the flat
// kernel, then the DFS kernel over the rows that were too much work for one
// thread (a star's match product, a chain walk's bucket rows).
static int run_flat_count(amj_ctx *ctx, ProbeLaunch &PL, ExecScratch &X, bool ws, uint64_t row_lo, uint64_t row_hi,
                          PassResult *pr, amj_result *res) {
    ProbePlan &P = PL.P;
    P.row_lo = row_lo;
    P.row_hi = row_hi;
    const uint64_t rows = row_hi - row_lo;
    struct Ctr {
        unsigned long long count, checksum;
        unsigned int nover, pad;
    };
    DBuf<Ctr> ctr;
    DBuf<uint32_t> over;
    AMJ_TRY(ctr.alloc(ctx, 1));
    AMJ_TRY(over.alloc(ctx, rows ? rows : 1));
    AMJ_CUDA_TRY(cudaMemsetAsync(ctr.p, 0, sizeof(Ctr), ctx->stream));
    const unsigned g = (unsigned)std::min<uint64_t>((rows + 255) / 256, (uint64_t)ctx->num_sms * 8);
    CanonPlan S{};
    int canon = star_canon(P, S);
    bool chain = false;
    if (!canon) {
        canon = chain_canon(P, S);
        chain = canon > 0;
    }
    DBuf<BucketHead> heads;
    uint32_t maxnb = 0;
    if (canon) {
        size_t tot = 0;
        for (int c = 0; c < canon; c++) {
            tot += S.nb[c];
            maxnb = std::max(maxnb, S.nb[c]);
        }
        // the heads (32 B a bucket, up to four times the levels' columns)
        // are built only while they take at most an eighth of the device's
        // memory; otherwise a star takes the general kernel and a chain the
        // DFS kernel
        if (tot * sizeof(BucketHead) > ctx->device_mem / 8) {
            if (chain) return run_passes(ctx, PL, X, ws, false, false, row_lo, row_hi, pr, res, false);
            canon = 0;
        } else {
            AMJ_TRY(heads.alloc(ctx, tot));
            // the heads are read by 256-bit loads, which need 32-byte alignment
            if (reinterpret_cast<uintptr_t>(heads.p) % alignof(BucketHead) != 0) {
                if (chain) return run_passes(ctx, PL, X, ws, false, false, row_lo, row_hi, pr, res, false);
                canon = 0;
            }
        }
    }
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[0], ctx->stream));
    if (canon) {
        HeadOut H{};
        size_t at = 0;
        for (int c = 0; c < canon; c++) {
            H.p[c] = heads.p + at;
            S.head[c] = heads.p + at;
            at += S.nb[c];
        }
        const unsigned gx = (unsigned)std::min<uint64_t>((maxnb + 255) / 256, (uint64_t)ctx->num_sms * 4);
        note_launch(ctx);
        bucket_heads_kernel<<<dim3(gx ? gx : 1, canon), 256, 0, ctx->stream>>>(S, H);
        AMJ_CUDA_TRY(cudaGetLastError());
    }
    note_launch(ctx);
    if (chain) {
        switch (canon) {
        case 1: amhj_chain_canon_kernel<1><<<g ? g : 1, 256, 0, ctx->stream>>>(S, &ctr.p->count, &ctr.p->checksum, over.p, &ctr.p->nover); break;
        case 2: amhj_chain_canon_kernel<2><<<g ? g : 1, 256, 0, ctx->stream>>>(S, &ctr.p->count, &ctr.p->checksum, over.p, &ctr.p->nover); break;
        case 3: amhj_chain_canon_kernel<3><<<g ? g : 1, 256, 0, ctx->stream>>>(S, &ctr.p->count, &ctr.p->checksum, over.p, &ctr.p->nover); break;
        case 4: amhj_chain_canon_kernel<4><<<g ? g : 1, 256, 0, ctx->stream>>>(S, &ctr.p->count, &ctr.p->checksum, over.p, &ctr.p->nover); break;
        case 5: amhj_chain_canon_kernel<5><<<g ? g : 1, 256, 0, ctx->stream>>>(S, &ctr.p->count, &ctr.p->checksum, over.p, &ctr.p->nover); break;
        default: amhj_chain_canon_kernel<6><<<g ? g : 1, 256, 0, ctx->stream>>>(S, &ctr.p->count, &ctr.p->checksum, over.p, &ctr.p->nover);
        }
    } else switch (canon) {
    case 1: amhj_star_canon_kernel<1><<<g ? g : 1, 256, 0, ctx->stream>>>(S, &ctr.p->count, &ctr.p->checksum, over.p, &ctr.p->nover); break;
    case 2: amhj_star_canon_kernel<2><<<g ? g : 1, 256, 0, ctx->stream>>>(S, &ctr.p->count, &ctr.p->checksum, over.p, &ctr.p->nover); break;
    case 3: amhj_star_canon_kernel<3><<<g ? g : 1, 256, 0, ctx->stream>>>(S, &ctr.p->count, &ctr.p->checksum, over.p, &ctr.p->nover); break;
    case 4: amhj_star_canon_kernel<4><<<g ? g : 1, 256, 0, ctx->stream>>>(S, &ctr.p->count, &ctr.p->checksum, over.p, &ctr.p->nover); break;
    default: amhj_star_kernel<<<g ? g : 1, 256, 0, ctx->stream>>>(P, &ctr.p->count, &ctr.p->checksum, over.p, &ctr.p->nover);
    }
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[1], ctx->stream));
    Ctr h{};
    AMJ_CUDA_TRY(cudaMemcpyAsync(&h, ctr.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    res->kernel_ms[0] += event_ms(ctx->kev[0], ctx->kev[1]);
    pr->count = h.count;
    pr->checksum = h.checksum;
    if (h.nover == 0) return AMJ_OK;
    // the listed rows, gathered into a probe relation of their own
    std::vector<DBuf<int32_t>> cols(P.probe_ncols);
    int32_t *cp[AMJ_MAX_COLS] = {};
    for (int c = 0; c < P.probe_ncols; c++) {
        AMJ_TRY(cols[c].alloc(ctx, h.nover));
        cp[c] = cols[c].p;
    }
    DBuf<int32_t *> dcp;
    AMJ_TRY(dcp.alloc(ctx, AMJ_MAX_COLS));
    AMJ_CUDA_TRY(cudaMemcpyAsync(dcp.p, cp, sizeof(cp), cudaMemcpyHostToDevice, ctx->stream));
    note_launch(ctx);
    star_gather_kernel<<<(unsigned)std::min<uint64_t>((h.nover + 255) / 256, (uint64_t)ctx->num_sms * 8), 256, 0,
                         ctx->stream>>>(P, over.p, h.nover, dcp.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    ProbeLaunch sub = PL;
    for (int c = 0; c < P.probe_ncols; c++) sub.P.probe_col[c] = cp[c];
    // The listed rows are the heavy ones, and gathered they sit in few warps'
    // row chunks: join them with work sharing whatever the query's ws, so
    // their frontiers spread over all warps (the same result).
    if (!ws) {
        if (!X.tasks.p) {
            AMJ_TRY(X.tasks.alloc(ctx, P.task_cap));
            AMJ_TRY(X.ready.alloc(ctx, P.task_cap));
        }
        sub.tasks = X.tasks.p;
        sub.task_ready = X.ready.p;
    }
    PassResult rest;
    AMJ_TRY(run_passes(ctx, sub, X, true, false, false, 0, h.nover, &rest, res, false));
    pr->count += rest.count;
    pr->checksum += rest.checksum;
    return AMJ_OK;
}

// Materialised star plan (dro=0): per-row tuple counts, a scan, exact
// allocation, and one flat write pass (amhj_star.cuh).
static int run_star_write(amj_ctx *ctx, ProbeLaunch &PL, uint64_t row_lo, uint64_t row_hi, PassResult *pr,
                          amj_result *res) {
    PL.P.row_lo = row_lo;
    PL.P.row_hi = row_hi;
    ProbePlan P = PL.P;
    const uint64_t rows = row_hi - row_lo;
    DBuf<unsigned long long> off, ctr;
    AMJ_TRY(off.alloc(ctx, rows + 1));
    AMJ_TRY(ctr.alloc(ctx, 2));
    const unsigned g = (unsigned)std::min<uint64_t>((rows + 255) / 256, (uint64_t)ctx->num_sms * 8);
    note_launch(ctx);
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[0], ctx->stream));
    star_rowcount_kernel<<<g ? g : 1, 256, 0, ctx->stream>>>(P, off.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[1], ctx->stream));
    AMJ_TRY(scan_exclusive_u64(ctx, (const uint64_t *)off.p, (uint64_t *)off.p, rows, (uint64_t *)off.p + rows));
    unsigned long long total = 0;
    AMJ_CUDA_TRY(cudaMemcpyAsync(&total, off.p + rows, sizeof(total), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    res->kernel_ms[0] += event_ms(ctx->kev[0], ctx->kev[1]);
    AMJ_TRY(alloc_cols(ctx, P.k, total, pr->cols));
    for (int a = 0; a < P.k; a++) P.out[a] = pr->cols[a];
    P.out_cap = total;
    AMJ_CUDA_TRY(cudaMemsetAsync(ctr.p, 0, 2 * sizeof(unsigned long long), ctx->stream));
    note_launch(ctx);
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[2], ctx->stream));
    star_write_kernel<<<g ? g : 1, 256, 0, ctx->stream>>>(P, off.p, ctr.p, ctr.p + 1);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_CUDA_TRY(cudaEventRecord(ctx->kev[3], ctx->stream));
    unsigned long long h[2] = {0, 0};
    AMJ_CUDA_TRY(cudaMemcpyAsync(h, ctr.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    res->kernel_ms[1] += event_ms(ctx->kev[2], ctx->kev[3]);
    if (h[0] != total) return fail(AMJ_ECUDA, "AMHJ: star write pass disagrees with its row counts");
    pr->count = total;
    pr->checksum = h[1];
    pr->rows = total;
    res->stats[3] += total;
    return AMJ_OK;
}

static int run_passes(amj_ctx *ctx, ProbeLaunch &PL, ExecScratch &X, bool ws, bool dro, bool materialize,
                      uint64_t row_lo, uint64_t row_hi, PassResult *pr, amj_result *res, bool allow_flat) {
    CanonPlan chain_shape;   // filled only to test the shape
    if (!materialize && allow_flat && (star_eligible(PL.P) || chain_canon(PL.P, chain_shape)))
        return run_flat_count(ctx, PL, X, ws, row_lo, row_hi, pr, res);
    if (materialize && !dro && allow_flat && star_eligible(PL.P))
        return run_star_write(ctx, PL, row_lo, row_hi, pr, res);
    ProbePlan &P = PL.P;
    P.row_lo = row_lo;
    P.row_hi = row_hi;
    const uint64_t rows = row_hi - row_lo;
    const uint64_t nbatches = (rows + 31) / 32;
    const uint32_t task_cap = ws ? P.task_cap : 0u;
    ProbeState h{};
    PL.batch_stride = 1;
    PL.batch_count = nbatches;
    const int k = P.k;
    // work sharing: balance level 0 by candidates instead of probe rows
    DBuf<unsigned long long> l0;
    P.lbs = 0;
    P.l0_start = nullptr;
    uint64_t nchunks = 0;
    if (ws && rows) {
        AMJ_TRY(l0.alloc(ctx, rows + 1));
        P.l0_start = l0.p;
        const unsigned g = (unsigned)std::min<uint64_t>((rows + 255) / 256, (uint64_t)ctx->num_sms * 16);
        note_launch(ctx);
        amhj_l0_sizes_kernel<<<g, 256, 0, ctx->stream>>>(P, l0.p);
        AMJ_CUDA_TRY(cudaGetLastError());
        AMJ_TRY(scan_exclusive_u64(ctx, (const uint64_t *)l0.p, (uint64_t *)l0.p, rows, (uint64_t *)l0.p + rows));
        unsigned long long total = 0;
        AMJ_CUDA_TRY(cudaMemcpyAsync(&total, l0.p + rows, sizeof(total), cudaMemcpyDeviceToHost, ctx->stream));
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        nchunks = (total + L0_CHUNK - 1) / L0_CHUNK;
        if (nchunks > 0xffffffffull) return fail(AMJ_EUNSUPPORTED, "AMHJ: more than 2^37 level-0 candidates in one slice");
        P.lbs = 1;
        PL.batch_count = nchunks;
    }

    if (!materialize) {
        P.dro = 0;
        AMJ_TRY(reset_state(ctx, PL.st, ws ? PL.task_ready : nullptr, task_cap));
        AMJ_TRY(launch_probe(ctx, PL, PM_COUNT, ws));
        AMJ_TRY(read_state(ctx, PL.st, &h, "AMHJ count", &res->kernel_ms[0]));
        pr->count = h.count;
        pr->checksum = h.checksum;
        res->stats[0] += h.tasks_pushed;
        res->stats[1] += h.tasks_popped;
        res->stats[10] += h.fib_rows;
        return AMJ_OK;
    }
    if (!dro) {
        // two passes: count, exact allocation, write (reference AMHJ_evaluate, AMHJ.cuh:314-377)
        P.dro = 0;
        AMJ_TRY(reset_state(ctx, PL.st, ws ? PL.task_ready : nullptr, task_cap));
        AMJ_TRY(launch_probe(ctx, PL, PM_COUNT, ws));
        AMJ_TRY(read_state(ctx, PL.st, &h, "AMHJ count", &res->kernel_ms[0]));
        const uint64_t total = h.count;
        res->stats[0] += h.tasks_pushed;
        res->stats[1] += h.tasks_popped;
        res->stats[10] += h.fib_rows;
        AMJ_TRY(alloc_cols(ctx, k, total, pr->cols));
        for (int a = 0; a < k; a++) P.out[a] = pr->cols[a];
        P.out_cap = total;
        AMJ_TRY(reset_state(ctx, PL.st, ws ? PL.task_ready : nullptr, task_cap));
        AMJ_TRY(launch_probe(ctx, PL, PM_WRITE, ws));
        AMJ_TRY(read_state(ctx, PL.st, &h, "AMHJ write", &res->kernel_ms[1]));
        if (h.count != total || h.out_cursor != total)
            return fail(AMJ_ECUDA, "AMHJ: write pass disagrees with count pass");
        pr->count = total;
        pr->checksum = h.checksum;
        pr->rows = total;
        res->stats[3] += total;
        return AMJ_OK;
    }
    // ---- direct result output (reference AMHJ_DRO, MHJ-GPU/Joins/AMHJ_DRO.cuh:506-707)
    // 1. estimate |OUT| by counting a strided sample of probe batches
    uint64_t estimate = 0;
    {
        const uint64_t want = 4096;   // batches sampled
        const uint64_t stride = nbatches > want ? nbatches / want : 1;
        P.dro = 0;
        const uint32_t lbs = P.lbs;
        P.lbs = 0;
        AMJ_TRY(reset_state(ctx, PL.st, nullptr, 0));
        PL.batch_stride = stride;
        PL.batch_count = (nbatches + stride - 1) / stride;
        AMJ_TRY(launch_probe(ctx, PL, PM_COUNT, false));
        AMJ_TRY(read_state(ctx, PL.st, &h, "AMHJ DRO sampling"));
        P.lbs = lbs;
        const double sampled_rows = std::min<double>((double)PL.batch_count * 32.0, (double)rows);
        const double est = sampled_rows > 0 ? (double)h.count * (double)rows / sampled_rows : 0.0;
        estimate = (uint64_t)(est * (ctx->opts.dro_headroom > 0.f ? ctx->opts.dro_headroom : 1.05f)) + 1024;
        PL.batch_stride = 1;
        PL.batch_count = P.lbs ? nchunks : nbatches;
    }
    res->stats[5] += estimate;
    // 2. one write pass into the estimated buffer, recording breakpoints
    int32_t *main_cols[AMJ_MAX_ATTRS] = {};
    AMJ_TRY(alloc_cols(ctx, k, estimate, main_cols));
    for (int a = 0; a < k; a++) P.out[a] = main_cols[a];
    P.out_cap = estimate;
    P.dro = 1;
    const uint64_t unit_cap = (P.lbs ? nchunks : nbatches) + task_cap + 64;
    if (X.units.n < unit_cap) AMJ_TRY(X.units.alloc(ctx, unit_cap));
    PL.units = X.units.p;
    P.unit_cap = (uint32_t)std::min<uint64_t>(unit_cap, 0xffffffffull);
    AMJ_TRY(reset_state(ctx, PL.st, ws ? PL.task_ready : nullptr, task_cap));
    int rc = launch_probe(ctx, PL, PM_WRITE, ws);
    if (rc == AMJ_OK) rc = read_state(ctx, PL.st, &h, "AMHJ DRO main write", &res->kernel_ms[1]);
    if (rc != AMJ_OK) {
        for (int a = 0; a < k; a++) dev_free(ctx, main_cols[a]);
        if (rc == AMJ_EOVERFLOW && ws) {
            // The residual replay needs every split of the main pass to have
            // reached the task queue; when the queue filled up, redo the
            // direct output without work sharing.
            AMJ_TRY(status_reset(ctx));
            res->stats[6]++;
            return run_passes(ctx, PL, X, false, dro, materialize, row_lo, row_hi, pr, res);
        }
        return rc;
    }
    const uint64_t total = h.count;
    const uint64_t written = std::min<uint64_t>(total, estimate);
    res->stats[0] += h.tasks_pushed;
    res->stats[1] += h.tasks_popped;
    res->stats[3] += written;
    pr->count = total;
    pr->checksum = h.checksum;
    pr->rows = total;
    if (total <= estimate) {
        for (int a = 0; a < k; a++) pr->cols[a] = main_cols[a];
        return AMJ_OK;
    }
    // 3. residual: resume the overflowed units after the rows they wrote
    const uint32_t n_units = h.n_units;
    res->stats[2] += n_units;
    rc = alloc_cols(ctx, k, total, pr->cols);
    if (rc != AMJ_OK) {
        for (int a = 0; a < k; a++) dev_free(ctx, main_cols[a]);
        return rc;
    }
    for (int a = 0; a < k; a++) {
        if (written)
            AMJ_CUDA_TRY(cudaMemcpyAsync(pr->cols[a], main_cols[a], written * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                                         ctx->stream));
        dev_free(ctx, main_cols[a]);
        P.out[a] = pr->cols[a] + written;
    }
    P.out_cap = total - written;
    P.dro = 0;
    // keep the task queue contents: the residual replays tasks by slot
    AMJ_CUDA_TRY(cudaMemsetAsync(PL.st, 0, sizeof(ProbeState), ctx->stream));
    PL.batch_count = n_units;
    AMJ_TRY(launch_probe(ctx, PL, PM_RESIDUAL, ws));
    AMJ_TRY(read_state(ctx, PL.st, &h, "AMHJ DRO residual write", &res->kernel_ms[1]));
    if (h.out_cursor != total - written)
        return fail(AMJ_ECUDA, "AMHJ DRO: residual pass wrote " + std::to_string(h.out_cursor) + " rows, expected " +
                                   std::to_string(total - written));
    res->stats[4] += h.out_cursor;
    return AMJ_OK;
}

// ---------------------------------------------------------------- FIB --
// Frequent-item buffering (reference AMHJ_WS_FIB, MHJ-GPU/Joins/AMHJ_WS_FIB.cuh,
// SubfixBuffer.cuh:65-98): the suffix of the query below some level d,
// when it depends on nothing but the key bound at d, is the same for every
// partial tuple arriving with the same key.  The frequent keys of level d
// (those of its largest buckets, read off the bucket index instead of a CPU
// Topkapi sketch) get their suffix tuples materialised once, by the same
// probe kernel run on a probe relation made of those keys; the main probe
// then emits a cached key's suffix tuples directly.  The checksum needs the
// tuples themselves (a tuple's hash chains its prefix into its suffix), so
// the cache holds tuples, not counts.

constexpr uint32_t FIB_MAX_KEYS = 256;
constexpr uint32_t FIB_MIN_BUCKET = 16;
constexpr uint64_t FIB_MAX_ROWS = 1ull << 26;

// the shallowest level d >= 1 with at least two levels below it whose suffix
// depends only on the key attribute of level d; -1 if none
static int fib_choose_level(const HostPlan &hp, uint32_t *suffix_attrs) {
    for (int d = 1; d + 1 < hp.L; d++) {
        const LevelSpec &ld = hp.lv[d];
        if (ld.key_mode != KEY_SINGLE) continue;
        const int ka = ld.attr[0];
        uint32_t suffix = 0;
        bool ok = true;
        for (int e = d; e < hp.L && ok; e++) {
            const LevelSpec &le = hp.lv[e];
            for (int c = 0; c < le.ncols; c++) {
                const int a = le.attr[c];
                if ((le.cmp_mask >> c) & 1) {
                    if (a != ka && !((suffix >> a) & 1)) ok = false;
                }
            }
            for (int c = 0; c < le.ncols; c++)
                if ((le.bind_mask >> c) & 1) suffix |= 1u << le.attr[c];
        }
        if (ok) {
            *suffix_attrs = suffix;
            return d;
        }
    }
    return -1;
}

__global__ void fib_bucket_sizes_kernel(const uint32_t *__restrict__ buc_ptrs, uint64_t B,
                                        uint64_t *__restrict__ items) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < B; b += (uint64_t)gridDim.x * blockDim.x)
        items[b] = ((uint64_t)(buc_ptrs[b + 1] - buc_ptrs[b]) << 32) | b;
}

__global__ void fib_first_keys_kernel(const uint64_t *__restrict__ items, uint32_t n,
                                      const uint32_t *__restrict__ buc_ptrs, const int32_t *__restrict__ key_col,
                                      int32_t *__restrict__ keys) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keys[i] = (items[i] >> 32) ? key_col[buc_ptrs[(uint32_t)items[i]]] : OA_EMPTY_KEY;
}

// cache index of every suffix tuple (via the key hash set), packed with its row
__global__ void fib_pack_kernel(const int32_t *__restrict__ key_col, uint64_t n, const int32_t *__restrict__ set_keys,
                                const uint32_t *__restrict__ set_idx, uint32_t mask, uint64_t *__restrict__ items,
                                unsigned long long *__restrict__ counts) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
        const int32_t key = key_col[r];
        uint32_t s = hash_key(key) & mask, idx = 0;
        for (uint32_t t = 0; t <= mask; t++) {
            if (set_keys[s] == key) {
                idx = set_idx[s];
                break;
            }
            s = (s + 1) & mask;
        }
        items[r] = ((uint64_t)idx << 32) | (uint32_t)r;
        atomicAdd(&counts[idx], 1ull);
    }
}

__global__ void fib_gather_kernel(const uint64_t *__restrict__ items, uint64_t n, const int32_t *__restrict__ src,
                                  int32_t *__restrict__ dst) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[(uint32_t)items[i]];
}

static unsigned fib_grid(amj_ctx *ctx, uint64_t n) {
    uint64_t g = (n + 255) / 256, cap = (uint64_t)ctx->num_sms * 16;
    return (unsigned)(g == 0 ? 1 : (g > cap ? cap : g));
}

static int build_fib(amj_ctx *ctx, const HostPlan &hp, const std::vector<const HashIndex *> &lvix, ProbeLaunch &PL,
                     ExecScratch &X, amj_result *res) {
    ProbePlan &P = PL.P;
    P.fib_level = -1;
    uint32_t suffix = 0;
    const int d = fib_choose_level(hp, &suffix);
    if (d < 0) return AMJ_OK;
    const HashIndex &ix = *lvix[d];
    if (ix.layout != AMJ_LAYOUT_BUCKET || ix.n < FIB_MIN_BUCKET) return AMJ_OK;
    // 1. frequent keys: first keys of the largest buckets
    const uint64_t B = (uint64_t)ix.mask + 1;
    DBuf<uint64_t> a, b;
    AMJ_TRY(a.alloc(ctx, B));
    AMJ_TRY(b.alloc(ctx, B));
    note_launch(ctx);
    fib_bucket_sizes_kernel<<<fib_grid(ctx, B), 256, 0, ctx->stream>>>(ix.buc_ptrs.p, B, a.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    uint64_t *sorted = nullptr;
    AMJ_TRY(radix_sort_u64(ctx, a.p, b.p, B, SK_IDENT, 32, 64, &sorted));
    const uint32_t take = (uint32_t)std::min<uint64_t>(B, FIB_MAX_KEYS);
    std::vector<uint64_t> top(take);
    AMJ_CUDA_TRY(cudaMemcpyAsync(top.data(), sorted + (B - take), take * 8, cudaMemcpyDeviceToHost, ctx->stream));
    DBuf<int32_t> keys_d;
    AMJ_TRY(keys_d.alloc(ctx, take));
    note_launch(ctx);
    fib_first_keys_kernel<<<(take + 255) / 256, 256, 0, ctx->stream>>>(sorted + (B - take), take, ix.buc_ptrs.p,
                                                                       ix.cols[0].p, keys_d.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    std::vector<int32_t> keys(take);
    AMJ_CUDA_TRY(cudaMemcpyAsync(keys.data(), keys_d.p, take * 4, cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    std::vector<int32_t> freq;
    for (uint32_t i = 0; i < take; i++)
        if ((top[i] >> 32) >= FIB_MIN_BUCKET && keys[i] != OA_EMPTY_KEY) freq.push_back(keys[i]);
    std::sort(freq.begin(), freq.end());
    freq.erase(std::unique(freq.begin(), freq.end()), freq.end());
    if (freq.empty()) return AMJ_OK;
    const uint32_t K = (uint32_t)freq.size();
    AMJ_CUDA_TRY(cudaMemcpyAsync(keys_d.p, freq.data(), K * 4, cudaMemcpyHostToDevice, ctx->stream));
    // 2. their suffix tuples: the sub-plan below level d probed by the keys
    ProbeLaunch SL = PL;
    ProbePlan &S = SL.P;
    S.L = (int8_t)(hp.L - d);
    for (int l = 0; l < S.L; l++) S.lv[l] = P.lv[d + l];
    S.probe_ncols = 1;
    S.probe_col[0] = keys_d.p;
    S.probe_attr[0] = (int8_t)hp.lv[d].attr[0];
    S.row_lo = 0;
    S.row_hi = K;
    S.warp_bytes = (uint32_t)S.L * S.depth_bytes;
    S.lbs = 0;
    S.dro = 0;
    S.fib_level = -1;
    plan_inline(S);
    SL.batch_stride = 1;
    SL.batch_count = (K + 31) / 32;
    ProbeState h{};
    AMJ_CUDA_TRY(cudaMemsetAsync(SL.st, 0, sizeof(ProbeState), ctx->stream));
    AMJ_TRY(launch_probe(ctx, SL, PM_COUNT, false));
    AMJ_TRY(read_state(ctx, SL.st, &h, "FIB suffix count"));
    const uint64_t T = h.count;
    if (T == 0 || T > FIB_MAX_ROWS) return AMJ_OK;
    const int k = hp.k;
    int32_t *tcols[AMJ_MAX_ATTRS] = {};
    std::vector<DBuf<int32_t>> tmp(k);
    for (int at = 0; at < k; at++) {
        AMJ_TRY(tmp[at].alloc(ctx, T));
        tcols[at] = tmp[at].p;
        S.out[at] = tcols[at];
    }
    S.out_cap = T;
    AMJ_CUDA_TRY(cudaMemsetAsync(SL.st, 0, sizeof(ProbeState), ctx->stream));
    AMJ_TRY(launch_probe(ctx, SL, PM_WRITE, false));
    AMJ_TRY(read_state(ctx, SL.st, &h, "FIB suffix write"));
    if (h.out_cursor != T) return fail(AMJ_ECUDA, "FIB: suffix write disagrees with its count");
    // 3. group the suffix tuples by key: hash set of the keys, sort by cache index
    uint32_t slots = 512;
    while (slots < 2 * K) slots <<= 1;
    std::vector<int32_t> skey(slots, OA_EMPTY_KEY);
    std::vector<uint32_t> sidx(slots, 0);
    for (uint32_t i = 0; i < K; i++) {
        uint32_t s = hash_key(freq[i]) & (slots - 1);
        while (skey[s] != OA_EMPTY_KEY) s = (s + 1) & (slots - 1);
        skey[s] = freq[i];
        sidx[s] = i;
    }
    AMJ_TRY(X.fib_keys.alloc(ctx, slots));
    AMJ_TRY(X.fib_idx.alloc(ctx, slots));
    AMJ_CUDA_TRY(cudaMemcpyAsync(X.fib_keys.p, skey.data(), slots * 4, cudaMemcpyHostToDevice, ctx->stream));
    AMJ_CUDA_TRY(cudaMemcpyAsync(X.fib_idx.p, sidx.data(), slots * 4, cudaMemcpyHostToDevice, ctx->stream));
    DBuf<uint64_t> ia, ib;
    DBuf<unsigned long long> counts;
    AMJ_TRY(ia.alloc(ctx, T));
    AMJ_TRY(ib.alloc(ctx, T));
    AMJ_TRY(counts.alloc(ctx, K));
    AMJ_CUDA_TRY(cudaMemsetAsync(counts.p, 0, K * 8, ctx->stream));
    note_launch(ctx);
    fib_pack_kernel<<<fib_grid(ctx, T), 256, 0, ctx->stream>>>(tcols[hp.lv[d].attr[0]], T, X.fib_keys.p, X.fib_idx.p,
                                                                slots - 1, ia.p, counts.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    uint64_t *by_key = nullptr;
    int kbits = 1;
    while ((1u << kbits) < K) kbits++;
    AMJ_TRY(radix_sort_u64(ctx, ia.p, ib.p, T, SK_IDENT, 32, 32 + kbits, &by_key));
    for (int at = 0; at < k; at++) {
        if (!((suffix >> at) & 1)) continue;
        AMJ_TRY(X.fib_cols[at].alloc(ctx, T));
        note_launch(ctx);
        fib_gather_kernel<<<fib_grid(ctx, T), 256, 0, ctx->stream>>>(by_key, T, tcols[at], X.fib_cols[at].p);
        AMJ_CUDA_TRY(cudaGetLastError());
        P.fib_cols[at] = X.fib_cols[at].p;
    }
    std::vector<unsigned long long> cnt(K), off(K + 1, 0);
    AMJ_CUDA_TRY(cudaMemcpyAsync(cnt.data(), counts.p, K * 8, cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (uint32_t i = 0; i < K; i++) off[i + 1] = off[i] + cnt[i];
    AMJ_TRY(X.fib_off.alloc(ctx, K + 1));
    AMJ_CUDA_TRY(cudaMemcpyAsync(X.fib_off.p, off.data(), (K + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    P.fib_keys = X.fib_keys.p;
    P.fib_slot_idx = X.fib_idx.p;
    P.fib_off = X.fib_off.p;
    P.fib_mask = slots - 1;
    P.fib_suffix_attrs = suffix;
    P.fib_level = d;
    res->stats[8] = K;
    res->stats[9] = T;
    return AMJ_OK;
}

void fill_level_desc(const LevelSpec &ls, int layout, int key_mode, uint32_t mask, const uint32_t *buc_ptrs,
                     const int32_t *const *cols, const int2 *slots, LevelDesc *d) {
    std::memset(d, 0, sizeof(*d));
    d->buc_ptrs = buc_ptrs;
    for (int c = 0; c < 4; c++) d->col[c] = cols[c];
    d->slots = slots;
    d->mask = mask;
    d->layout = (int8_t)layout;
    d->key_mode = (int8_t)key_mode;
    d->ncols = (int8_t)ls.ncols;
    d->key_attr[0] = (int8_t)ls.attr[0];
    d->key_attr[1] = (int8_t)(ls.ncols > 1 ? ls.attr[1] : 0);
    d->cmp_mask = ls.cmp_mask;
    d->bind_mask = ls.bind_mask;
    for (int c = 0; c < 4; c++) d->attr[c] = (int8_t)(c < ls.ncols ? ls.attr[c] : 0);
}

void fill_level_from_index(const LevelSpec &ls, const HashIndex &ix, LevelDesc *d) {
    const int32_t *cols[4] = {ix.cols[0].p, ix.cols[1].p, ix.cols[2].p, ix.cols[3].p};
    fill_level_desc(ls, ix.layout, ix.key_mode, ix.mask, ix.buc_ptrs.p, cols, ix.slots.p, d);
}

static void fill_level(const LevelSpec &ls, const HashIndex &ix, LevelDesc *d) { fill_level_from_index(ls, ix, d); }

void plan_common(const HostPlan &hp, const amj_opts &o, ProbePlan *P) {
    P->L = (int8_t)hp.L;
    P->k = (int8_t)hp.k;
    P->probe_ncols = (int8_t)hp.probe->ncols;
    for (int c = 0; c < hp.probe->ncols && c < AMJ_MAX_COLS; c++) {
        P->probe_col[c] = hp.probe->d_cols[c];
        P->probe_attr[c] = (int8_t)hp.probe_attr[c];
    }
    P->task_chunk = (uint32_t)o.task_chunk;
    P->task_cap = (uint32_t)std::min<uint64_t>(o.task_capacity, 0x7fffffffull);
    P->spin_limit_ns = (uint64_t)o.spin_limit_ms * 1000000ull;
    P->depth_bytes = frontier_bytes(hp.k);
    P->warp_bytes = (uint32_t)hp.L * P->depth_bytes;
    P->fib_level = -1;
}

// ---- out-of-core (reference OOC::execute ooc=1, MHJ-GPU/ooc.cuh:166-306) ----
// The probe relation is processed in slices.  When it lives in host memory
// (AMJ_MEM_HOST_STREAMED) each slice is copied into one of two device staging
// buffers on a side stream while the previous slice is joined, and the
// materialised rows of every slice go back to host memory, so neither the
// input nor the output has to fit on the device.  Build relations stay
// resident, as in the reference.
int amhj_ooc_execute(amj_ctx *ctx, ProbeLaunch &PL, ExecScratch *X, const amj_rel *probe, bool ws, bool dro,
                     bool materialize, int flags, amj_result *out) {
    const int nc = probe->ncols;
    const uint64_t n = probe->n;
    const bool host = probe->where == AMJ_MEM_HOST_STREAMED;
    uint64_t slice = ctx->opts.ooc_slice_rows;
    if (!slice) {
        size_t fr = 0, tot = 0;
        AMJ_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        const uint64_t budget = ctx->opts.mem_budget ? ctx->opts.mem_budget : fr / 2;
        slice = budget / 8 / ((uint64_t)nc * 4);
    }
    slice = std::max<uint64_t>(1024, (slice + 31) / 32 * 32);
    const uint64_t nslices = n ? (n + slice - 1) / slice : 0;
    const int k = PL.P.k;

    DBuf<int32_t> stage[2][AMJ_MAX_COLS];
    cudaEvent_t ready[2] = {nullptr, nullptr};
    bool registered[AMJ_MAX_COLS] = {};
    auto cleanup = [&]() {
        for (int b = 0; b < 2; b++)
            if (ready[b]) cudaEventDestroy(ready[b]);
        for (int c = 0; c < nc; c++)
            if (registered[c]) cudaHostUnregister((void *)probe->h_cols[c]);
        (void)cudaGetLastError();
    };
    if (host) {
        for (int b = 0; b < 2; b++) {
            for (int c = 0; c < nc; c++) {
                int rc = stage[b][c].alloc(ctx, std::min<uint64_t>(slice, n ? n : 1));
                if (rc != AMJ_OK) { cleanup(); return rc; }
            }
            if (cudaEventCreateWithFlags(&ready[b], cudaEventDisableTiming) != cudaSuccess) {
                cleanup();
                return fail(AMJ_ECUDA, "ooc: event creation failed");
            }
        }
        // page-lock the caller's columns so the staging copies run asynchronously
        for (int c = 0; c < nc; c++)
            registered[c] = cudaHostRegister((void *)probe->h_cols[c], n * sizeof(int32_t),
                                             cudaHostRegisterReadOnly) == cudaSuccess;
        (void)cudaGetLastError();
        // the staging buffers are stream-ordered allocations of the context
        // stream; the side stream may write them only after they exist
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            cleanup();
            return fail(AMJ_ECUDA, "ooc: synchronising the staging allocations failed");
        }
    }
    auto stage_copy = [&](uint64_t s) -> int {
        const int b = (int)(s & 1);
        const uint64_t lo = s * slice, hi = std::min(n, lo + slice);
        for (int c = 0; c < nc; c++)
            AMJ_CUDA_TRY(cudaMemcpyAsync(stage[b][c].p, probe->h_cols[c] + lo, (hi - lo) * sizeof(int32_t),
                                         cudaMemcpyHostToDevice, ctx->side_stream[0]));
        AMJ_CUDA_TRY(cudaEventRecord(ready[b], ctx->side_stream[0]));
        return AMJ_OK;
    };
    std::vector<std::vector<int32_t>> hcols(materialize ? k : 0);
    uint64_t count = 0, checksum = 0;
    int rc = AMJ_OK;
    if (host && nslices) rc = stage_copy(0);
    for (uint64_t s = 0; rc == AMJ_OK && s < nslices; s++) {
        const uint64_t lo = s * slice, hi = std::min(n, lo + slice);
        uint64_t rlo = lo, rhi = hi;
        if (host) {
            const int b = (int)(s & 1);
            rc = cudaStreamWaitEvent(ctx->stream, ready[b], 0) == cudaSuccess ? AMJ_OK : AMJ_ECUDA;
            if (rc != AMJ_OK) break;
            for (int c = 0; c < nc; c++) PL.P.probe_col[c] = stage[b][c].p;
            rlo = 0;
            rhi = hi - lo;
            // the other buffer was last read by slice s-1, which has completed
            if (s + 1 < nslices) rc = stage_copy(s + 1);
            if (rc != AMJ_OK) break;
        }
        PassResult pr;
        rc = run_passes(ctx, PL, *X, ws, dro, materialize, rlo, rhi, &pr, out, !(flags & AMJ_F_FRONTIER));
        if (rc != AMJ_OK) break;
        count += pr.count;
        checksum += pr.checksum;
        if (materialize) {
            for (int a = 0; a < k && rc == AMJ_OK; a++) {
                const size_t old = hcols[a].size();
                hcols[a].resize(old + pr.rows);
                if (pr.rows && cudaMemcpyAsync(hcols[a].data() + old, pr.cols[a], pr.rows * sizeof(int32_t),
                                               cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
                    rc = fail(AMJ_ECUDA, "ooc: result copy failed");
            }
            if (rc == AMJ_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = fail(AMJ_ECUDA, "ooc: sync failed");
            for (int a = 0; a < k; a++) dev_free(ctx, pr.cols[a]);
        }
    }
    // no staging copy may outlive its buffer, on the error paths too
    if (host) (void)cudaStreamSynchronize(ctx->side_stream[0]);
    cleanup();
    if (rc != AMJ_OK) return rc;
    out->count = count;
    out->checksum = checksum;
    out->stats[7] = nslices;
    if (materialize) {
        auto *o = new ResultOwner();
        o->ctx = ctx;
        out->priv = o;
        out->on_host = 1;
        out->rows = count;
        for (int a = 0; a < k; a++) {
            if (cudaMallocHost((void **)&out->cols[a], (count ? count : 1) * sizeof(int32_t)) != cudaSuccess) {
                (void)cudaGetLastError();
                return fail(AMJ_ENOMEM, "ooc: pinned result allocation failed");
            }
            if (count) std::memcpy(out->cols[a], hcols[a].data(), count * sizeof(int32_t));
        }
    }
    return AMJ_OK;
}

}  // namespace amj

using namespace amj;

extern "C" int amj_amhj_execute(amj_ctx *ctx, int query_type, amj_rel *const *rels, int nrels, int ooc, int ws,
                                int dro, int fib, int flags, amj_result *out) {
    if (!ctx || !out || !rels || nrels <= 0) return fail(AMJ_EINVAL, "amhj_execute: bad arguments");
    for (int i = 0; i < nrels; i++)
        if (!rels[i]) return fail(AMJ_EINVAL, "amhj_execute: null relation");
    AMJ_CUDA_TRY(cudaSetDevice(ctx->device));
    // TRI / FOUR over one edge relation: the pair-key levels through a
    // bitmap of b's children (TRI) or the triangle matrices (FOUR) of the
    // degree-ranked copy, where they apply
    if ((query_type == AMJ_QUERY_TRI || query_type == AMJ_QUERY_FOUR) && nrels == 1 && rels[0]->ncols == 2 &&
        rels[0]->where != AMJ_MEM_HOST_STREAMED && !ooc &&
        !(flags & (AMJ_F_KEEP_ORDER | AMJ_F_HASH_PLAN | AMJ_F_THREAD_PER_ROW | AMJ_F_PAIRWISE))) {
        bool used = false;
        if (query_type == AMJ_QUERY_TRI) AMJ_TRY(amhj_tri_by_wedges(ctx, rels[0], flags, out, &used));
        else AMJ_TRY(amhj_four_by_matrices(ctx, rels[0], flags, out, &used));
        if (used) return AMJ_OK;
        amj_result_release(out);
    }
    // TRI / FOUR over an oriented edge relation: join its degree-ordered copy
    // and report every tuple sorted (the same bag; shorter hub lists)
    amj_rel ordered;
    amj_rel *ordered_rels[1] = {&ordered};
    DBuf<int32_t> ord0, ord1;
    bool sort_out = false;
    if ((query_type == AMJ_QUERY_TRI || query_type == AMJ_QUERY_FOUR) && nrels == 1 && rels[0]->ncols == 2 &&
        rels[0]->where != AMJ_MEM_HOST_STREAMED && !(flags & AMJ_F_KEEP_ORDER)) {
        AMJ_TRY(degree_ordered_copy(ctx, rels[0]->d_cols[0], rels[0]->d_cols[1], rels[0]->n, &ord0, &ord1,
                                    &sort_out));
        if (sort_out) {
            ordered = *rels[0];
            ordered.uid = 0;   // a temporary relation: never kept by an index provider
            ordered.owned = false;
            ordered.d_cols[0] = ord0.p;
            ordered.d_cols[1] = ord1.p;
            rels = ordered_rels;
        }
    }
    HostPlan hp;
    AMJ_TRY(compile_plan(query_type, rels, nrels, flags, &hp));
    result_init(out, hp.k);
    const bool materialize = (flags & AMJ_F_MATERIALIZE) != 0;
    // frequent-item buffering runs on the work-sharing kernel (reference
    // AMHJ_WS_FIB, exec_AMHJ.cu:171-176)
    const bool use_ws = ws != 0 || fib != 0;
    const int layout = ctx->opts.layout;

    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1], e2 = ctx->ev[2];
    AMJ_CUDA_TRY(cudaEventRecord(e0, ctx->stream));

    if (flags & AMJ_F_PAIRWISE) {
        if (query_type != AMJ_QUERY_NORMAL || hp.L < 1 || ooc || fib)
            return fail(AMJ_EUNSUPPORTED, "amhj_execute: the pairwise plan takes NORMAL queries, ooc=0, fib=0");
        for (int i = 0; i < nrels; i++)
            if (rels[i]->where == AMJ_MEM_HOST_STREAMED) return fail(AMJ_EUNSUPPORTED, "pairwise plan: device relations");
        const auto t0 = std::chrono::steady_clock::now();
        int rc = amhj_pairwise_execute(ctx, hp, ws, dro, flags & ~AMJ_F_HOST_RESULT, out);
        if (rc != AMJ_OK) {
            amj_result_release(out);
            return rc;
        }
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        out->total_ms = out->probe_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        out->build_ms = 0;
        if (materialize) {
            rc = finish_result_columns(ctx, out, flags);
            if (rc != AMJ_OK) {
                amj_result_release(out);
                return rc;
            }
        }
        return AMJ_OK;
    }
    bool host_builds = false;
    for (int i = 1; i < nrels; i++) host_builds |= rels[i]->where == AMJ_MEM_HOST_STREAMED;
    if (rels[0]->where == AMJ_MEM_HOST_STREAMED && !ooc)
        return fail(AMJ_EINVAL, "amhj_execute: a relation kept on the host needs ooc=1");
    if (host_builds) {
        // build relations in host memory: the staged, partitioned form
        if (!ooc) return fail(AMJ_EINVAL, "amhj_execute: a relation kept on the host needs ooc=1");
        if (query_type != AMJ_QUERY_NORMAL || hp.L == 0)
            return fail(AMJ_EUNSUPPORTED, "amhj_execute: host-resident build relations need a NORMAL query");
        // the part joins reuse the context's events: time the stages on the host
        const auto t0 = std::chrono::steady_clock::now();
        int rc = amhj_partitioned_execute(ctx, hp, use_ws ? 1 : 0, dro, flags, out);
        if (rc != AMJ_OK) {
            amj_result_release(out);
            return rc;
        }
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        out->total_ms = out->probe_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (materialize) {
            rc = finish_result_columns(ctx, out, flags);
            if (rc != AMJ_OK) {
                amj_result_release(out);
                return rc;
            }
        }
        return AMJ_OK;
    }

    ExecScratch X;
    // ---- build phase
    std::vector<const HashIndex *> lvix(hp.L);
    for (int l = 0; l < hp.L; l++) {
        const LevelSpec &ls = hp.lv[l];
        IndexKey key{ls.rel, {-1, -1, -1, -1}, ls.ncols, ls.key_mode, layout};
        for (int c = 0; c < ls.ncols; c++) key.src[c] = ls.src_col[c];
        key.uid = ls.rel->uid;
        key.load_factor = ctx->opts.load_factor;
        if (ctx->iprov && ls.rel->uid) {
            if (const HashIndex *kept = ctx->iprov->get(ctx, key, ls)) {
                lvix[l] = kept;
                continue;
            }
        }
        auto it = X.indexes.find(key);
        if (it == X.indexes.end()) {
            HashIndex ix;
            const int32_t *cols[4];
            for (int c = 0; c < ls.ncols; c++) cols[c] = ls.rel->d_cols[ls.src_col[c]];
            int rc = build_hash_index(ctx, cols, ls.ncols, ls.rel->n, layout, ls.key_mode, ctx->opts.load_factor, &ix);
            if (rc != AMJ_OK && layout == AMJ_LAYOUT_CUCKOO && rc == AMJ_EOVERFLOW) {
                // more copies of a key than two cuckoo buckets hold: bucket layout for this table
                ix = HashIndex();
                rc = build_hash_index(ctx, cols, ls.ncols, ls.rel->n, AMJ_LAYOUT_BUCKET, ls.key_mode,
                                      ctx->opts.load_factor, &ix);
                out->stats[6]++;
            }
            if (rc != AMJ_OK) return rc;
            it = X.indexes.emplace(key, std::move(ix)).first;
        }
        lvix[l] = &it->second;
    }
    AMJ_CUDA_TRY(cudaEventRecord(e1, ctx->stream));

    // ---- probe plan
    ProbeLaunch PL;
    std::memset(&PL, 0, sizeof(PL));
    ProbePlan &P = PL.P;
    plan_common(hp, ctx->opts, &P);
    for (int l = 0; l < hp.L; l++) fill_level(hp.lv[l], *lvix[l], &P.lv[l]);
    plan_inline(P);
    P.sort_out = sort_out ? 1 : 0;
    AMJ_TRY(X.st.alloc(ctx, 1));
    PL.st = X.st.p;
    PL.status = ctx->d_status;
    if (use_ws) {
        AMJ_TRY(X.tasks.alloc(ctx, P.task_cap));
        AMJ_TRY(X.ready.alloc(ctx, P.task_cap));
        PL.tasks = X.tasks.p;
        PL.task_ready = X.ready.p;
    }
    AMJ_TRY(status_reset(ctx));
    if (fib && !dro && hp.L >= 3) AMJ_TRY(build_fib(ctx, hp, lvix, PL, X, out));

    int rc = AMJ_OK;
    if (hp.L == 0) {
        // a single relation: the result is the relation itself
        const amj_rel *r = hp.probe;
        if (r->where == AMJ_MEM_HOST_STREAMED) return fail(AMJ_EUNSUPPORTED, "amhj_execute: single host relation");
        std::vector<int32_t> tmp;
        out->count = r->n;
        std::vector<std::vector<int32_t>> hcols(hp.k, std::vector<int32_t>(r->n));
        for (int c = 0; c < r->ncols; c++)
            AMJ_CUDA_TRY(cudaMemcpyAsync(hcols[hp.probe_attr[c]].data(), r->d_cols[c], r->n * 4, cudaMemcpyDeviceToHost,
                                         ctx->stream));
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        std::vector<const int32_t *> cp(hp.k);
        for (int a = 0; a < hp.k; a++) cp[a] = hcols[a].data();
        AMJ_TRY(amj_checksum_host(cp.data(), hp.k, r->n, &out->checksum));
        if (materialize) {
            int32_t *cols[AMJ_MAX_ATTRS] = {};
            AMJ_TRY(alloc_cols(ctx, hp.k, r->n, cols));
            for (int c = 0; c < r->ncols; c++)
                AMJ_CUDA_TRY(cudaMemcpyAsync(cols[hp.probe_attr[c]], r->d_cols[c], r->n * 4, cudaMemcpyDeviceToDevice,
                                             ctx->stream));
            auto *o = new ResultOwner();
            o->ctx = ctx;
            out->priv = o;
            for (int a = 0; a < hp.k; a++) out->cols[a] = cols[a];
            out->rows = r->n;
        }
    } else if (ooc || hp.probe->where == AMJ_MEM_HOST_STREAMED) {
        rc = amhj_ooc_execute(ctx, PL, &X, hp.probe, use_ws, dro != 0, materialize, flags, out);
    } else if (flags & AMJ_F_THREAD_PER_ROW) {
        // the thread-per-row baseline (count only)
        if (materialize || !thread_row_eligible(P)) {
            rc = fail(AMJ_EUNSUPPORTED, "amhj_execute: the thread-per-row baseline counts over bucket indexes only");
        } else {
            DBuf<unsigned long long> c2;
            rc = c2.alloc(ctx, 2);
            if (rc == AMJ_OK && cudaMemsetAsync(c2.p, 0, 16, ctx->stream) != cudaSuccess)
                rc = fail(AMJ_ECUDA, "thread-per-row: memset");
            if (rc == AMJ_OK) {
                P.row_lo = 0;
                P.row_hi = hp.probe->n;
                const uint64_t n = hp.probe->n;
                note_launch(ctx);
                (void)cudaEventRecord(ctx->kev[0], ctx->stream);
                amhj_thread_row_kernel<<<(unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256,
                                                                                             (uint64_t)ctx->num_sms * 8)),
                                         256, 0, ctx->stream>>>(P, c2.p, c2.p + 1);
                (void)cudaEventRecord(ctx->kev[1], ctx->stream);
                unsigned long long h2[2] = {0, 0};
                if (cudaGetLastError() != cudaSuccess ||
                    cudaMemcpyAsync(h2, c2.p, 16, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
                    cudaStreamSynchronize(ctx->stream) != cudaSuccess)
                    rc = fail(AMJ_ECUDA, "thread-per-row kernel");
                out->count = h2[0];
                out->checksum = h2[1];
                out->kernel_ms[0] = event_ms(ctx->kev[0], ctx->kev[1]);
            }
        }
    } else {
        PassResult pr;
        rc = run_passes(ctx, PL, X, use_ws, dro != 0, materialize, 0, hp.probe->n, &pr, out, !(flags & AMJ_F_FRONTIER));
        if (rc == AMJ_OK) {
            out->count = pr.count;
            out->checksum = pr.checksum;
            if (materialize) {
                auto *o = new ResultOwner();
                o->ctx = ctx;
                out->priv = o;
                for (int a = 0; a < hp.k; a++) out->cols[a] = pr.cols[a];
                out->rows = pr.rows;
            }
        }
    }
    if (rc != AMJ_OK) {
        amj_result_release(out);
        return rc;
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
