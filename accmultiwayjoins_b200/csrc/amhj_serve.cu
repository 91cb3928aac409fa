// Request server: a loop over relations kept resident in HBM that admits AMHJ
// queries by device memory and runs them by continuous batching.
//
// No reference counterpart (the reference runs one query per process).  A
// host thread owns the device work:
//  * lanes: each lane is a context with its own stream.  A free lane takes
//    the waiting requests in arrival order (up to max_batch, and only while
//    their estimated device memory fits the budget left by the batches in
//    flight) and launches them as one batch on a share of the SMs, then the
//    loop goes on; requests that arrive meanwhile are admitted into the next
//    free lane, so batches overlap on the device.  A finished lane publishes
//    its requests' results and returns its memory to the budget.
//  * the out-of-core lane: requests whose relations stay in host memory
//    (AMJ_MEM_HOST_STREAMED) and requests too large for the whole budget
//    (spilled) run through the ooc operator, which streams probe slices from
//    pinned host buffers on its side stream, on a context and a host thread
//    of their own, next to the batches.
// Every wait is bounded: a batch that does not finish within the spin limit
// of its kernels is reported by the kernels themselves (AMJ_ETIMEOUT).
#include "amhj_batch.h"

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

using namespace amj;

namespace {

struct ServeReq {
    uint64_t id = 0;
    int qt = 0, flags = 0;
    std::vector<amj_rel *> rels;
    bool ooc = false;
    uint64_t need = 0;               // estimated device bytes in a batch
    double t_submit = 0, t_start = 0, t_done = 0;
    uint64_t count = 0, checksum = 0;
    int status = AMJ_OK;
    int path = 0;                    // 0 batch, 1 out-of-core lane
    int state = 0;                   // 0 waiting, 1 running, 2 done
    uint32_t batch_id = 0, batch_size = 0;
    bool spilled = false;
    std::string error;               // message of a failed request
};

// Indexes of the resident relations, kept for the server's lifetime and
// shared by its lanes and its out-of-core lane: a request whose build
// relations were indexed before only probes.  An index is built on the first
// miss, on the calling lane's stream, and synchronised before anyone uses it;
// keys carry the relation's serial number, so a released relation's address
// reused by a new one never hits.  Indexes that would exceed the capacity
// are not kept (the batch builds them as usual).
struct ServerIndexCache : IndexProvider {
    std::mutex mu;
    std::map<IndexKey, std::unique_ptr<HashIndex>> kept;
    std::map<IndexKey, int> refused;
    uint64_t bytes = 0, cap = 0, hits = 0, builds = 0;

    static uint64_t index_bytes(const HashIndex &ix) {
        uint64_t b = ix.buc_ptrs.n * sizeof(uint32_t) + ix.slots.n * sizeof(int2);
        for (const auto &c : ix.cols) b += c.n * sizeof(int32_t);
        return b;
    }

    const HashIndex *get(amj_ctx *ctx, const IndexKey &key, const LevelSpec &ls) override {
        std::lock_guard<std::mutex> lk(mu);
        auto it = kept.find(key);
        if (it != kept.end()) {
            hits++;
            return it->second.get();
        }
        if (refused.count(key)) return nullptr;
        const uint64_t n = ls.rel->n;
        const double lf = key.load_factor > 0.f ? key.load_factor : 0.5;
        const uint64_t est = n * 4ull * ls.ncols + (uint64_t)((double)n / lf) * 8 + 4096;
        if (bytes + est > cap) {
            refused[key] = 1;
            return nullptr;
        }
        auto ix = std::make_unique<HashIndex>();
        const int32_t *cols[4] = {nullptr, nullptr, nullptr, nullptr};
        for (int c = 0; c < ls.ncols; c++) cols[c] = ls.rel->d_cols[ls.src_col[c]];
        int rc = build_hash_index(ctx, cols, ls.ncols, n, key.layout, ls.key_mode, key.load_factor, ix.get());
        if (rc == AMJ_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = AMJ_ECUDA;
        if (rc != AMJ_OK) {
            (void)cudaGetLastError();
            refused[key] = 1;
            return nullptr;
        }
        builds++;
        bytes += index_bytes(*ix);
        const HashIndex *p = ix.get();
        kept.emplace(key, std::move(ix));
        return p;
    }
};

struct Lane {
    amj_ctx *ctx = nullptr;
    amj_batch *b = nullptr;
    std::vector<ServeReq *> reqs;
    uint64_t reserved = 0;
    uint32_t batch_id = 0;
    bool busy = false;
};

}  // namespace

struct amj_server {
    amj_ctx *main = nullptr;
    amj_serve_opts opts{};
    amj_batch_opts bopts{};
    std::vector<Lane> lanes;
    amj_ctx *ooc_ctx = nullptr;
    std::thread loop, ooc_loop;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_ooc;
    std::deque<ServeReq *> pending, ooc_pending;
    std::unordered_map<uint64_t, std::unique_ptr<ServeReq>> reqs;
    uint64_t next_id = 1;
    uint64_t budget = 0, reserved = 0, peak_reserved = 0;
    bool stop = false;
    std::chrono::steady_clock::time_point t0;
    amj_serve_stats st{};
    uint32_t inflight = 0;
    std::unique_ptr<ServerIndexCache> cache;

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

// Estimated device bytes of one request inside a batch.
uint64_t request_bytes(const HostPlan &hp, const amj_batch_opts &o) {
    const double lf = o.load_factor > 0.f ? o.load_factor : 1.0;
    uint64_t rows = 0, buckets = 0;
    for (int l = 0; l < hp.L; l++) {
        rows += hp.lv[l].rel->n;
        buckets += (uint64_t)((double)hp.lv[l].rel->n / lf) + 1;
    }
    return rows * 33 + buckets * (o.layout == AMJ_LAYOUT_OPEN_ADDR ? 16 : 4) + hp.probe->n * 16 + 4096;
}

void finish(amj_server *s, ServeReq *r, int status) {
    r->status = status;
    if (status != AMJ_OK && r->error.empty()) {
        const char *m = amj_last_error();   // the failing call ran on this thread
        r->error = m ? m : "";
    }
    r->t_done = s->now();
    r->state = 2;
    s->st.completed++;
}

// Launch the requests of one lane as a batch.  Called without the lock.  The
// lane's batch object is reused: its device and pinned buffers only grow.
int launch_lane(amj_server *s, Lane &ln) {
    batch_clear(ln.b);
    for (ServeReq *r : ln.reqs)
        AMJ_TRY(amj_batch_submit(ln.b, r->qt, r->rels.data(), (int)r->rels.size(), r->flags & AMJ_F_NO_REORDER,
                                 nullptr));
    return batch_launch(ln.b, s->bopts);
}

void server_loop(amj_server *s) {
    cudaSetDevice(s->main->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        // ---- finished lanes publish their results
        for (Lane &ln : s->lanes) {
            if (!ln.busy || !batch_done(ln.b)) continue;
            lk.unlock();
            std::vector<uint64_t> cnt(ln.reqs.size()), chk(ln.reqs.size());
            const int rc = batch_collect(ln.b, cnt.data(), chk.data(), nullptr);
            lk.lock();
            for (size_t i = 0; i < ln.reqs.size(); i++) {
                ln.reqs[i]->count = cnt[i];
                ln.reqs[i]->checksum = chk[i];
                finish(s, ln.reqs[i], rc);
            }
            ln.reqs.clear();
            s->reserved -= ln.reserved;
            ln.reserved = 0;
            ln.busy = false;
            s->inflight--;
            s->cv_done.notify_all();
        }
        bool any_busy = false;
        for (Lane &ln : s->lanes) any_busy |= ln.busy;
        if (s->stop && s->pending.empty() && !any_busy) break;

        // ---- free lanes admit waiting requests
        for (Lane &ln : s->lanes) {
            if (ln.busy || s->pending.empty()) continue;
            uint64_t take = 0;
            while (!s->pending.empty() && ln.reqs.size() < s->opts.max_batch) {
                ServeReq *r = s->pending.front();
                if (r->need > s->budget) {
                    // too large for the device budget even alone: out-of-core
                    // lane, or rejected when the server has none
                    s->pending.pop_front();
                    if (!s->opts.ooc_lane) {
                        s->st.rejected++;
                        r->error = "the request needs more device memory than the whole budget, and the server "
                                   "has no out-of-core lane";
                        finish(s, r, AMJ_EREJECT);
                        s->cv_done.notify_all();
                        continue;
                    }
                    r->spilled = true;
                    r->ooc = true;
                    s->st.spilled++;
                    s->ooc_pending.push_back(r);
                    s->cv_ooc.notify_one();
                    continue;
                }
                if (s->reserved + take + r->need > s->budget) break;   // wait for memory
                s->pending.pop_front();
                take += r->need;
                ln.reqs.push_back(r);
            }
            if (ln.reqs.empty()) break;
            const double t = s->now();
            for (ServeReq *r : ln.reqs) {
                r->state = 1;
                r->t_start = t;
                r->batch_id = (uint32_t)s->st.batches;
                r->batch_size = (uint32_t)ln.reqs.size();
            }
            ln.batch_id = (uint32_t)s->st.batches++;
            ln.reserved = take;
            s->reserved += take;
            if (s->reserved > s->peak_reserved) s->peak_reserved = s->reserved;
            ln.busy = true;
            s->inflight++;
            if (s->inflight > s->st.max_inflight_batches) s->st.max_inflight_batches = s->inflight;
            lk.unlock();
            const int rc = launch_lane(s, ln);
            lk.lock();
            if (rc != AMJ_OK) {
                for (ServeReq *r : ln.reqs) finish(s, r, rc);
                ln.reqs.clear();
                s->reserved -= ln.reserved;
                ln.reserved = 0;
                ln.busy = false;
                s->inflight--;
                s->cv_done.notify_all();
            }
        }
        // ---- sleep until a request arrives or, with batches in flight, poll again shortly
        any_busy = false;
        for (Lane &ln : s->lanes) any_busy |= ln.busy;
        if (any_busy) s->cv_work.wait_for(lk, std::chrono::microseconds(50));
        else if (!s->stop) s->cv_work.wait_for(lk, std::chrono::milliseconds(20));
    }
}

void server_ooc_loop(amj_server *s) {
    cudaSetDevice(s->main->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        if (s->ooc_pending.empty()) {
            if (s->stop && s->pending.empty()) {
                bool any_busy = false;
                for (Lane &ln : s->lanes) any_busy |= ln.busy;
                if (!any_busy) break;
            }
            s->cv_ooc.wait_for(lk, std::chrono::milliseconds(20));
            continue;
        }
        ServeReq *r = s->ooc_pending.front();
        s->ooc_pending.pop_front();
        r->state = 1;
        r->path = 1;
        r->t_start = s->now();
        lk.unlock();
        amj_result res;
        std::memset(&res, 0, sizeof(res));
        const int rc = amj_amhj_execute(s->ooc_ctx, r->qt, r->rels.data(), (int)r->rels.size(), 1, 1, 0, 0,
                                        r->flags & AMJ_F_NO_REORDER, &res);
        lk.lock();
        r->count = res.count;
        r->checksum = res.checksum;
        if (rc == AMJ_OK) amj_result_release(&res);
        s->st.ooc_runs++;
        finish(s, r, rc);
        s->cv_done.notify_all();
    }
}

}  // namespace

extern "C" int amj_server_create(amj_ctx *ctx, const amj_serve_opts *opts, amj_server **out) {
    if (!ctx || !out) return fail(AMJ_EINVAL, "server_create: null argument");
    auto s = std::make_unique<amj_server>();
    s->main = ctx;
    if (opts) s->opts = *opts;
    if (s->opts.lanes <= 0) s->opts.lanes = 2;
    if (s->opts.lanes > 16) return fail(AMJ_EINVAL, "server_create: at most 16 lanes");
    if (s->opts.max_batch == 0) s->opts.max_batch = 256;
    AMJ_TRY(normalize_batch_opts(&s->opts.batch, &s->bopts));
    s->bopts.use_graph = 0;   // every batch is a new mix: eager launches
    AMJ_CUDA_TRY(cudaSetDevice(ctx->device));
    size_t fr = 0, tot = 0;
    AMJ_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    uint64_t ooc_reserve = 0;
    if (s->opts.ooc_lane) ooc_reserve = s->opts.ooc_mem ? s->opts.ooc_mem : (uint64_t)(fr / 8);
    uint64_t cache_cap = 0;
    if (!s->opts.no_index_cache) cache_cap = s->opts.index_cache_bytes ? s->opts.index_cache_bytes : (uint64_t)(fr * 0.35);
    const uint64_t reserved0 = ooc_reserve + cache_cap;
    s->budget = s->opts.mem_budget ? s->opts.mem_budget
                                   : ((uint64_t)(fr * 0.8) > reserved0 ? (uint64_t)(fr * 0.8) - reserved0 : fr / 16);
    if (cache_cap) {
        s->cache = std::make_unique<ServerIndexCache>();
        s->cache->cap = cache_cap;
    }
    // The persistent kernels of the lanes and of the ooc lane run at the same
    // time; their idle warps wait for their own unstarted blocks, so all of
    // them must be resident together.  Each gets an equal share of four probe
    // blocks per SM: with the default 256-thread blocks (at most 64 registers
    // a thread, frontiers of at most 61 KB for a batch of 8-attribute queries
    // and 29 KB for an ooc chain) one block of each fits an SM together.
    int sms = 0;
    AMJ_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const int kernels = s->opts.lanes + (s->opts.ooc_lane ? 1 : 0);
    const int share = std::max(1, 4 / kernels) * sms;
    if (s->bopts.grid_blocks == 0 && kernels > 1) s->bopts.grid_blocks = share;
    amj_opts lo = ctx->opts;
    for (int i = 0; i < s->opts.lanes; i++) {
        Lane ln;
        int rc = amj_ctx_create(ctx->device, &lo, &ln.ctx);
        if (rc == AMJ_OK) rc = amj_batch_create(ln.ctx, &ln.b);
        if (rc == AMJ_OK) ln.ctx->iprov = s->cache.get();
        if (rc != AMJ_OK) {
            if (ln.ctx) amj_ctx_destroy(ln.ctx);
            for (Lane &l : s->lanes) {
                amj_batch_destroy(l.b);
                amj_ctx_destroy(l.ctx);
            }
            return rc;
        }
        s->lanes.push_back(ln);
    }
    if (s->opts.ooc_lane) {
        amj_opts oo = ctx->opts;
        oo.mem_budget = ooc_reserve;
        if (kernels > 1 && oo.max_blocks == 0) oo.max_blocks = (uint32_t)share;
        if (s->opts.ooc_slice_rows) oo.ooc_slice_rows = s->opts.ooc_slice_rows;
        int rc = amj_ctx_create(ctx->device, &oo, &s->ooc_ctx);
        if (rc == AMJ_OK) s->ooc_ctx->iprov = s->cache.get();
        if (rc != AMJ_OK) {
            for (Lane &l : s->lanes) {
                amj_batch_destroy(l.b);
                amj_ctx_destroy(l.ctx);
            }
            return rc;
        }
    }
    s->t0 = std::chrono::steady_clock::now();
    amj_server *raw = s.release();
    raw->loop = std::thread(server_loop, raw);
    if (raw->opts.ooc_lane) raw->ooc_loop = std::thread(server_ooc_loop, raw);
    *out = raw;
    return AMJ_OK;
}

extern "C" int amj_server_submit(amj_server *s, int query_type, amj_rel *const *rels, int nrels, int flags,
                                 int ooc, uint64_t *ticket) {
    if (!s || !rels || nrels <= 0 || !ticket) return fail(AMJ_EINVAL, "server_submit: bad arguments");
    if (flags & ~AMJ_F_NO_REORDER) return fail(AMJ_EUNSUPPORTED, "server_submit: served queries count only");
    bool host = false;
    for (int i = 0; i < nrels; i++) {
        if (!rels[i]) return fail(AMJ_EINVAL, "server_submit: null relation");
        if (rels[i]->ctx->device != s->main->device) return fail(AMJ_EINVAL, "server_submit: relation on another device");
        host |= rels[i]->where == AMJ_MEM_HOST_STREAMED;
    }
    auto r = std::make_unique<ServeReq>();
    HostPlan hp;
    AMJ_TRY(compile_plan(query_type, rels, nrels, flags, &hp));
    if (hp.L == 0) return fail(AMJ_EUNSUPPORTED, "server_submit: a query needs at least one build relation");
    r->qt = query_type;
    r->flags = flags;
    r->rels.assign(rels, rels + nrels);
    r->ooc = ooc != 0 || host;
    r->need = request_bytes(hp, s->bopts);
    if (r->ooc && !s->opts.ooc_lane) return fail(AMJ_EUNSUPPORTED, "server_submit: the server has no out-of-core lane");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail(AMJ_EINVAL, "server_submit: server is stopping");
    r->id = s->next_id++;
    r->t_submit = s->now();
    ServeReq *p = r.get();
    s->reqs.emplace(p->id, std::move(r));
    s->st.submitted++;
    if (p->ooc) {
        s->ooc_pending.push_back(p);
        s->cv_ooc.notify_one();
    } else {
        s->pending.push_back(p);
        s->cv_work.notify_one();
    }
    *ticket = p->id;
    return AMJ_OK;
}

extern "C" int amj_server_wait(amj_server *s, uint64_t ticket, uint32_t timeout_ms, amj_serve_result *out) {
    if (!s || !out) return fail(AMJ_EINVAL, "server_wait: null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(AMJ_EINVAL, "server_wait: unknown ticket");
    ServeReq *r = it->second.get();
    const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->state == 2; });
    if (!ok) return fail(AMJ_ETIMEOUT, "server_wait: request not finished within the timeout");
    std::memset(out, 0, sizeof(*out));
    out->count = r->count;
    out->checksum = r->checksum;
    out->status = r->status;
    out->path = r->path;
    out->spilled = r->spilled ? 1 : 0;
    out->queue_ms = (r->t_start - r->t_submit) * 1e3;
    out->exec_ms = (r->t_done - r->t_start) * 1e3;
    out->latency_ms = (r->t_done - r->t_submit) * 1e3;
    out->batch_id = r->batch_id;
    out->batch_size = r->batch_size;
    const int status = r->status;
    const std::string err = r->error;
    s->reqs.erase(it);
    if (status != AMJ_OK) return fail(status, "server_wait: the request failed: " + err);
    return AMJ_OK;
}

extern "C" int amj_server_stats(amj_server *s, amj_serve_stats *out) {
    if (!s || !out) return fail(AMJ_EINVAL, "server_stats: null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->budget_bytes = s->budget;
    out->peak_reserved_bytes = s->peak_reserved;
    out->launches = 0;
    for (const Lane &ln : s->lanes) out->launches += ln.ctx->launches;
    if (s->ooc_ctx) out->launches += s->ooc_ctx->launches;
    if (s->cache) {
        std::lock_guard<std::mutex> ck(s->cache->mu);
        out->index_hits = s->cache->hits;
        out->index_builds = s->cache->builds;
        out->index_bytes = s->cache->bytes;
    }
    out->lanes = (uint32_t)s->lanes.size();
    return AMJ_OK;
}

extern "C" int amj_server_destroy(amj_server *s) {
    if (!s) return AMJ_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_ooc.notify_all();
    if (s->loop.joinable()) s->loop.join();
    if (s->ooc_loop.joinable()) s->ooc_loop.join();
    for (Lane &ln : s->lanes)
        if (ln.b) amj_batch_destroy(ln.b);
    // the kept indexes were allocated on the lanes' contexts: free them first
    if (s->cache) {
        for (Lane &ln : s->lanes) cudaStreamSynchronize(ln.ctx->stream);
        if (s->ooc_ctx) cudaStreamSynchronize(s->ooc_ctx->stream);
        s->cache.reset();
    }
    for (Lane &ln : s->lanes) amj_ctx_destroy(ln.ctx);
    if (s->ooc_ctx) amj_ctx_destroy(s->ooc_ctx);
    delete s;
    return AMJ_OK;
}
