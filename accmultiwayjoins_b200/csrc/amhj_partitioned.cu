// AMHJ out-of-core when the build relations live in host memory too.
//
// The reference's ooc=1 (OOC::execute, MHJ-GPU/ooc.cuh:166-306) slices only
// the probe relation: every build relation and its hash table must fit on
// the device (amhj_ooc_execute does the same).  When build relations are kept
// in host memory (AMJ_MEM_HOST_STREAMED), the join runs here in stages, one
// per build relation in plan order, as a Grace hash join generalised to the
// multi-way plan:
//   stage j joins the intermediate result I (the probe relation at stage 0)
//   with build relation B_j on B_j's key attribute, which I binds.  Both are
//   hash-partitioned on the key into P parts (P a power of two chosen so one
//   part of each fits the memory budget: opts.mem_budget, else half the free
//   device memory); part p of I can only match part p of B_j.  Each pair is
//   copied to the device and joined by the 2-relation AMHJ operator (every
//   bound attribute compared, as in the full plan).  The rows of every stage
//   but the last go back to host memory and form the next intermediate; the
//   last stage sums counts and checksums (and collects the rows when asked).
// Every result tuple of the full plan is produced exactly once: its key at
// stage j puts it in exactly one part.  The relations of a stage are
// renamed to attributes 0..m-1 in id order, which leaves the last stage's
// tuples (all attributes) in attribute-id order, so its checksum is the
// query's.
#include "amhj_host.h"

#include <omp.h>

#include <algorithm>
#include <cstring>
#include <vector>

namespace amj {

namespace {

// A host relation: columns in attribute order `attrs`.
struct HostTable {
    std::vector<int> attrs;
    std::vector<std::vector<int32_t>> cols;
    uint64_t n = 0;
};

// Hash partition of n rows (columns cols) on column kc into P parts: the
// rows of part p are out[c][off[p] .. off[p+1]).
void partition_rows(const std::vector<const int32_t *> &cols, uint64_t n, int kc, uint32_t P,
                    std::vector<std::vector<int32_t>> *out, std::vector<uint64_t> *off) {
    const int nc = (int)cols.size();
    out->assign(nc, std::vector<int32_t>(n));
    off->assign(P + 1, 0);
    if (P == 1) {
        for (int c = 0; c < nc; c++)
            if (n) std::memcpy((*out)[c].data(), cols[c], n * 4);
        (*off)[1] = n;
        return;
    }
    const int T = n < (1u << 16) ? 1 : omp_get_max_threads();
    std::vector<uint64_t> cnt((size_t)T * P, 0);
    const int32_t *key = cols[kc];
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const uint64_t lo = n * t / T, hi = n * (t + 1) / T;
        uint64_t *mine = cnt.data() + (size_t)t * P;
        for (uint64_t i = lo; i < hi; i++) mine[hash_key(key[i]) & (P - 1)]++;
#pragma omp barrier
#pragma omp single
        {
            uint64_t acc = 0;
            for (uint32_t p = 0; p < P; p++) {
                (*off)[p] = acc;
                for (int u = 0; u < T; u++) {
                    const uint64_t c = cnt[(size_t)u * P + p];
                    cnt[(size_t)u * P + p] = acc;
                    acc += c;
                }
            }
            (*off)[P] = acc;
        }
        for (uint64_t i = lo; i < hi; i++) {
            const uint64_t pos = mine[hash_key(key[i]) & (P - 1)]++;
            for (int c = 0; c < nc; c++) (*out)[c][pos] = cols[c][i];
        }
    }
}

uint32_t parts_for(uint64_t bytes, uint64_t budget) {
    uint64_t p = 1;
    while (p < (1u << 20) && bytes > budget * p) p <<= 1;
    return (uint32_t)p;
}

}  // namespace

int amhj_partitioned_execute(amj_ctx *ctx, const HostPlan &hp, int ws, int dro, int flags, amj_result *out) {
    uint64_t budget = ctx->opts.mem_budget;
    if (!budget) {
        size_t fr = 0, tot = 0;
        AMJ_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        budget = fr / 2;
    }
    const bool materialize = (flags & AMJ_F_MATERIALIZE) != 0;
    // stage 0's intermediate: the probe relation (host or device columns)
    HostTable I;
    const amj_rel *pr = hp.probe;
    I.n = pr->n;
    std::vector<const int32_t *> icols;
    for (int c = 0; c < pr->ncols; c++) {
        I.attrs.push_back(hp.probe_attr[c]);
        if (pr->where == AMJ_MEM_HOST_STREAMED) {
            icols.push_back(pr->h_cols[c]);
        } else {
            I.cols.emplace_back(pr->n);
            if (pr->n)
                AMJ_CUDA_TRY(cudaMemcpyAsync(I.cols.back().data(), pr->d_cols[c], pr->n * 4, cudaMemcpyDeviceToHost,
                                             ctx->stream));
        }
    }
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (pr->where != AMJ_MEM_HOST_STREAMED)
        for (auto &c : I.cols) icols.push_back(c.data());
    uint64_t count = 0, checksum = 0, joins = 0;
    std::vector<std::vector<int32_t>> final_cols(materialize ? hp.k : 0);
    for (int j = 0; j < hp.L; j++) {
        const LevelSpec &ls = hp.lv[j];
        const amj_rel *B = ls.rel;
        const bool last = j + 1 == hp.L;
        // the stage's attributes, renamed to 0..m-1 in id order
        std::vector<int> S = I.attrs;
        for (int c = 0; c < B->ncols; c++) S.push_back((int)B->attrs[c]);
        std::sort(S.begin(), S.end());
        S.erase(std::unique(S.begin(), S.end()), S.end());
        auto rename = [&](int a) { return (uint32_t)(std::lower_bound(S.begin(), S.end(), a) - S.begin()); };
        const int ka = ls.attr[0];
        const int ik = (int)(std::find(I.attrs.begin(), I.attrs.end(), ka) - I.attrs.begin());
        if (ik == (int)I.attrs.size()) return fail(AMJ_EUNSUPPORTED, "AMHJ ooc: a build key the plan does not bind");
        std::vector<const int32_t *> bcols;
        for (int c = 0; c < B->ncols; c++) bcols.push_back(B->where == AMJ_MEM_HOST_STREAMED ? B->h_cols[c] : nullptr);
        std::vector<std::vector<int32_t>> bhost;
        if (B->where != AMJ_MEM_HOST_STREAMED) {
            bhost.assign(B->ncols, std::vector<int32_t>(B->n));
            for (int c = 0; c < B->ncols; c++) {
                if (B->n)
                    AMJ_CUDA_TRY(cudaMemcpyAsync(bhost[c].data(), B->d_cols[c], B->n * 4, cudaMemcpyDeviceToHost,
                                                 ctx->stream));
                bcols[c] = bhost[c].data();
            }
            AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        }
        // a part of each side within the budget: the probe part's columns, the
        // build part's columns and its index (about three times its columns)
        const uint64_t bytes = I.n * 4 * I.attrs.size() + B->n * 4 * (uint64_t)B->ncols * 4;
        const uint32_t P = parts_for(bytes, budget);
        std::vector<std::vector<int32_t>> ip, bp;
        std::vector<uint64_t> ioff, boff;
        partition_rows(icols, I.n, ik, P, &ip, &ioff);
        partition_rows(bcols, B->n, ls.src_col[0], P, &bp, &boff);
        HostTable next;
        next.attrs = S;
        next.cols.assign(S.size(), {});
        uint32_t pattrs[AMJ_MAX_COLS], battrs[AMJ_MAX_COLS];
        for (size_t c = 0; c < I.attrs.size(); c++) pattrs[c] = rename(I.attrs[c]);
        for (int c = 0; c < B->ncols; c++) battrs[c] = rename((int)B->attrs[c]);
        for (uint32_t p = 0; p < P; p++) {
            const uint64_t np = ioff[p + 1] - ioff[p], nb = boff[p + 1] - boff[p];
            if (np == 0 || nb == 0) continue;
            const int32_t *pc[AMJ_MAX_COLS], *bc[AMJ_MAX_COLS];
            for (size_t c = 0; c < I.attrs.size(); c++) pc[c] = ip[c].data() + ioff[p];
            for (int c = 0; c < B->ncols; c++) bc[c] = bp[c].data() + boff[p];
            amj_rel *rp = nullptr, *rb = nullptr;
            AMJ_TRY(amj_rel_create(ctx, np, (int)I.attrs.size(), pattrs, pc, AMJ_MEM_HOST, &rp));
            int rc = amj_rel_create(ctx, nb, B->ncols, battrs, bc, AMJ_MEM_HOST, &rb);
            amj_result res;
            std::memset(&res, 0, sizeof(res));
            const int f = (last && !materialize) ? 0 : (AMJ_F_MATERIALIZE | AMJ_F_HOST_RESULT);
            amj_rel *pair[2] = {rp, rb};
            if (rc == AMJ_OK) rc = amj_amhj_execute(ctx, AMJ_QUERY_NORMAL, pair, 2, 0, ws, dro, 0, f, &res);
            if (rc == AMJ_OK) {
                joins++;
                if (last) {
                    count += res.count;
                    checksum += res.checksum;
                }
                if (f) {
                    std::vector<std::vector<int32_t>> &dst = last ? final_cols : next.cols;
                    for (size_t a = 0; a < S.size(); a++) {
                        const size_t old = dst[a].size();
                        dst[a].resize(old + res.rows);
                        if (res.rows) std::memcpy(dst[a].data() + old, res.cols[a], res.rows * 4);
                    }
                    if (!last) next.n += res.rows;
                }
                amj_result_release(&res);
            }
            amj_rel_release(rp);
            if (rb) amj_rel_release(rb);
            if (rc != AMJ_OK) return rc;
        }
        if (!last) {
            I = std::move(next);
            icols.clear();
            for (auto &c : I.cols) icols.push_back(c.data());
        }
    }
    out->count = count;
    out->checksum = checksum;
    out->stats[7] = joins;   // partition pairs joined
    if (materialize) {
        auto *o = new ResultOwner();
        o->ctx = ctx;
        out->priv = o;
        out->rows = count;
        out->on_host = 1;
        for (int a = 0; a < hp.k; a++) {
            if (cudaMallocHost((void **)&out->cols[a], (count ? count : 1) * 4) != cudaSuccess) {
                (void)cudaGetLastError();
                return fail(AMJ_ENOMEM, "AMHJ ooc: pinned result allocation failed");
            }
            if (count) std::memcpy(out->cols[a], final_cols[a].data(), count * 4);
        }
    }
    return AMJ_OK;
}

// ---- pairwise baseline (AMJ_F_PAIRWISE) ----
// The plan as a chain of 2-relation joins on the device, each intermediate
// result materialised before the next join: the binary-join plan a
// multi-way join is compared with (the reference's exec_PW.cu runs such
// plans with a pairwise radix join).  Attributes are renamed per join as in
// the staged form above.
int amhj_pairwise_execute(amj_ctx *ctx, const HostPlan &hp, int ws, int dro, int flags, amj_result *out) {
    const bool materialize = (flags & AMJ_F_MATERIALIZE) != 0;
    amj_rel cur = *hp.probe;
    cur.uid = 0;
    cur.owned = false;
    for (int c = 0; c < cur.ncols; c++) cur.attrs[c] = (uint32_t)hp.probe_attr[c];
    amj_result prev;
    bool have_prev = false;
    int rc = AMJ_OK;
    for (int j = 0; j < hp.L && rc == AMJ_OK; j++) {
        const amj_rel *B = hp.lv[j].rel;
        const bool last = j + 1 == hp.L;
        std::vector<int> S;
        for (int c = 0; c < cur.ncols; c++) S.push_back((int)cur.attrs[c]);
        for (int c = 0; c < B->ncols; c++) S.push_back((int)B->attrs[c]);
        std::sort(S.begin(), S.end());
        S.erase(std::unique(S.begin(), S.end()), S.end());
        auto rename = [&](int a) { return (uint32_t)(std::lower_bound(S.begin(), S.end(), a) - S.begin()); };
        amj_rel pv = cur, bv = *B;
        bv.uid = 0;
        bv.owned = false;
        for (int c = 0; c < pv.ncols; c++) pv.attrs[c] = rename((int)cur.attrs[c]);
        for (int c = 0; c < bv.ncols; c++) bv.attrs[c] = rename((int)B->attrs[c]);
        amj_rel *pair[2] = {&pv, &bv};
        amj_result res;
        std::memset(&res, 0, sizeof(res));
        const int f = last ? (materialize ? AMJ_F_MATERIALIZE : 0) : AMJ_F_MATERIALIZE;
        rc = amj_amhj_execute(ctx, AMJ_QUERY_NORMAL, pair, 2, 0, ws, dro, 0, f, &res);
        if (rc != AMJ_OK) break;
        if (have_prev) amj_result_release(&prev);
        prev = res;
        have_prev = true;
        if (last) break;
        // the next probe relation: this join's rows, on the device
        cur = amj_rel();
        cur.ctx = ctx;
        cur.n = res.rows;
        cur.ncols = (int)S.size();
        cur.where = AMJ_MEM_DEVICE;
        for (size_t a = 0; a < S.size(); a++) {
            cur.attrs[a] = (uint32_t)S[a];
            cur.d_cols[a] = res.cols[a];
        }
    }
    if (rc != AMJ_OK) {
        if (have_prev) amj_result_release(&prev);
        return rc;
    }
    const int k = out->num_attrs;
    *out = prev;   // the last join's result, columns (when kept) on the device
    out->num_attrs = k;
    out->stats[7] = (uint64_t)hp.L;
    return AMJ_OK;
}

}  // namespace amj
