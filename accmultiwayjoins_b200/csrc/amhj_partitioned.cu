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
//   part of each, twice for the double buffer, and B_j's index fit the
//   memory budget: opts.mem_budget, else half the free device memory); part
//   p of I can only match part p of B_j.  Each pair is copied to the device
//   and joined by the 2-relation AMHJ operator (every bound attribute
//   compared, as in the full plan).  The rows of every stage but the last go
//   back to host memory and form the next intermediate; the last stage sums
//   counts and checksums (and collects the rows when asked).
// Every result tuple of the full plan is produced exactly once: its key at
// stage j puts it in exactly one part.  The relations of a stage are
// renamed to attributes 0..m-1 in id order, which leaves the last stage's
// tuples (all attributes) in attribute-id order, so its checksum is the
// query's.
//
// Host memory: the partitions and intermediates live in pinned blocks that
// the context keeps after the call (pinning tens of GB takes seconds, and a
// served system runs the same stages again); amj_ctx_trim and the context's
// destruction free them.  Rows are grouped by key hash on the device (input
// tables stream through it in chunks; each part result is grouped before it
// is copied back), so a part is a union of groups and the host scatters
// nothing up to 256 parts.  Part p+1 is copied to the device on one side
// stream while part p is joined, and part p's grouped result goes back on
// the other side stream while part p+1 is joined.
#include "amhj_host.h"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <vector>

namespace amj {

// ---- pinned host blocks kept by the context ----
struct PinnedCache {
    std::multimap<size_t, void *> free_blocks;   // by size
};

namespace {

size_t pinned_round(size_t b) {
    const size_t g = b <= (64ull << 20) ? (1ull << 20) : (64ull << 20);
    return (b + g - 1) / g * g;
}

PinnedCache *pinned_cache(amj_ctx *ctx) {
    if (!ctx->pinned_cache) ctx->pinned_cache = new PinnedCache();
    return static_cast<PinnedCache *>(ctx->pinned_cache);
}

void pinned_trim(amj_ctx *ctx) {
    PinnedCache *pc = pinned_cache(ctx);
    for (auto &kv : pc->free_blocks) (void)cudaFreeHost(kv.second);
    pc->free_blocks.clear();
}

// A pinned block of at least `bytes`: a kept block of up to 4/3 the rounded
// request, else a new one (after dropping the kept ones if pinning fails).
// Kept blocks are not dropped on a miss: pinning is slow (dropping them
// whenever they could not serve a request made a 3.4 s staged join take
// 27 s), so they stay until amj_ctx_trim or the context's end.
int pinned_get(amj_ctx *ctx, size_t bytes, void **p, size_t *size) {
    PinnedCache *pc = pinned_cache(ctx);
    const size_t r = pinned_round(bytes ? bytes : 1);
    auto it = pc->free_blocks.lower_bound(r);
    if (it != pc->free_blocks.end() && it->first <= r + r / 3) {
        *p = it->second;
        *size = it->first;
        pc->free_blocks.erase(it);
        return AMJ_OK;
    }
    cudaError_t e = cudaHostAlloc(p, r, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        pinned_trim(ctx);
        e = cudaHostAlloc(p, r, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            *p = nullptr;
            return fail(AMJ_ENOMEM, "AMHJ ooc: pinned host allocation of " + std::to_string(r) + " bytes failed");
        }
    }
    *size = r;
    return AMJ_OK;
}

// A pinned block, back to the context's cache when dropped.
struct Pinned {
    amj_ctx *ctx = nullptr;
    void *p = nullptr;
    size_t size = 0;
    Pinned() = default;
    Pinned(const Pinned &) = delete;
    Pinned &operator=(const Pinned &) = delete;
    Pinned(Pinned &&o) noexcept : ctx(o.ctx), p(o.p), size(o.size) { o.p = nullptr; }
    int get(amj_ctx *c, size_t bytes) {
        drop();
        ctx = c;
        return pinned_get(c, bytes, &p, &size);
    }
    void drop() {
        if (p) pinned_cache(ctx)->free_blocks.emplace(size, p);
        p = nullptr;
    }
    int32_t *i32() const { return static_cast<int32_t *>(p); }
    ~Pinned() { drop(); }
};

// Rows of a host table: pieces, each with one pointer per column.
struct Piece {
    const int32_t *col[AMJ_MAX_COLS] = {};
    uint64_t n = 0;
};

struct HostTable {
    std::vector<int> attrs;
    std::vector<Piece> pieces;
    std::vector<Pinned> own;   // pinned blocks holding the pieces (intermediates)
    uint64_t n = 0;
    // rows already grouped on the device by hash_key(column sub_col) &
    // (SUB_PARTS - 1): sub[s] lists the pieces of group s (also in `pieces`)
    int sub_col = -1;
    std::vector<std::vector<Piece>> sub;
};

// ---- grouping a part's result rows on the device ----
// The rows a stage returns form the next stage's intermediate, which is
// partitioned on the next key.  They are grouped on the device into
// SUB_PARTS groups by that key's hash before they are copied back, so that
// a part of the next stage (P <= SUB_PARTS parts, P a power of two) is the
// union of the groups s with s & (P - 1) == p, and the host scatters
// nothing.  One count pass, a scan of the counts, then tiles of rows
// scattered with one atomic reservation per group and tile.
constexpr uint32_t SUB_PARTS = 256;
constexpr uint32_t SUB_TILE = 4096;

struct SubCols {
    const int32_t *src[AMJ_MAX_ATTRS];
    int nc;
    int kc;
};

__global__ void sub_count_kernel(const int32_t *__restrict__ key, uint64_t n, unsigned int *__restrict__ cnt) {
    __shared__ unsigned int h[SUB_PARTS];
    for (uint32_t i = threadIdx.x; i < SUB_PARTS; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&h[hash_key(key[i]) & (SUB_PARTS - 1)], 1u);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < SUB_PARTS; i += blockDim.x)
        if (h[i]) atomicAdd(&cnt[i], h[i]);
}

// cursor[s]: the next free row of group s in dst (column c at dst + c * n)
__global__ void sub_scatter_kernel(const SubCols C, uint64_t n, unsigned int *__restrict__ cursor,
                                   int32_t *__restrict__ dst) {
    __shared__ unsigned int h[SUB_PARTS], base[SUB_PARTS];
    for (uint64_t t0 = (uint64_t)blockIdx.x * SUB_TILE; t0 < n; t0 += (uint64_t)gridDim.x * SUB_TILE) {
        for (uint32_t i = threadIdx.x; i < SUB_PARTS; i += blockDim.x) h[i] = 0;
        __syncthreads();
        const uint64_t t1 = t0 + SUB_TILE < n ? t0 + SUB_TILE : n;
        constexpr int IPT = SUB_TILE / 256;
        uint32_t grp[IPT], rk[IPT];
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const uint64_t i = t0 + (uint64_t)k * blockDim.x + threadIdx.x;
            if (i < t1) {
                grp[k] = hash_key(C.src[C.kc][i]) & (SUB_PARTS - 1);
                rk[k] = atomicAdd(&h[grp[k]], 1u);
            }
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < SUB_PARTS; i += blockDim.x)
            base[i] = h[i] ? atomicAdd(&cursor[i], h[i]) : 0u;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const uint64_t i = t0 + (uint64_t)k * blockDim.x + threadIdx.x;
            if (i < t1) {
                const uint64_t pos = (uint64_t)base[grp[k]] + rk[k];
                for (int c = 0; c < C.nc; c++) dst[(uint64_t)c * n + pos] = C.src[c][i];
            }
        }
        __syncthreads();
    }
}

// A table hash-partitioned on one column: part p is a list of pieces.
struct Parts {
    std::vector<std::vector<Piece>> part;
    std::vector<uint64_t> rows;
    Pinned block;
    uint64_t max_rows = 0;
};

// Hash partition of X on column kc into P parts, on all host cores: one
// counting pass, then every column scattered into one pinned block (column
// c of part p at c * n + off[p]).  P = 1 keeps X's pieces.
int partition_table(amj_ctx *ctx, const HostTable &X, int kc, uint32_t P, Parts *out) {
    out->part.assign(P, {});
    out->rows.assign(P, 0);
    out->max_rows = 0;
    const uint64_t n = X.n;
    if (P == 1) {
        for (const Piece &pc : X.pieces)
            if (pc.n) out->part[0].push_back(pc);
        out->rows[0] = out->max_rows = n;
        return AMJ_OK;
    }
    if (X.sub_col == kc && P <= SUB_PARTS && X.sub.size() == SUB_PARTS) {
        // grouped on the device already: part p is the union of its groups
        for (uint32_t g = 0; g < SUB_PARTS; g++)
            for (const Piece &pc : X.sub[g]) {
                out->part[g & (P - 1)].push_back(pc);
                out->rows[g & (P - 1)] += pc.n;
            }
        for (uint32_t p = 0; p < P; p++) out->max_rows = std::max(out->max_rows, out->rows[p]);
        return AMJ_OK;
    }
    if (n == 0) return AMJ_OK;
    const int nc = (int)X.attrs.size();
    AMJ_TRY(out->block.get(ctx, (size_t)nc * n * sizeof(int32_t)));
    int32_t *base = out->block.i32();
    std::vector<uint64_t> start(X.pieces.size() + 1, 0);   // first row of every piece
    for (size_t i = 0; i < X.pieces.size(); i++) start[i + 1] = start[i] + X.pieces[i].n;
    const int T = n < (1u << 16) ? 1 : omp_get_max_threads();
    std::vector<uint64_t> cnt((size_t)T * P, 0);
    std::vector<uint64_t> off(P + 1, 0);
    // rows [lo, hi) of the concatenated pieces, piece by piece
    auto for_range = [&](uint64_t lo, uint64_t hi, auto &&f) {
        size_t i = std::upper_bound(start.begin(), start.end(), lo) - start.begin() - 1;
        for (; lo < hi && i < X.pieces.size(); i++) {
            const uint64_t e = std::min(hi, start[i + 1]);
            if (e > lo) f(X.pieces[i], lo - start[i], e - start[i]);
            lo = e;
        }
    };
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const uint64_t lo = n * t / T, hi = n * (t + 1) / T;
        uint64_t *mine = cnt.data() + (size_t)t * P;
        for_range(lo, hi, [&](const Piece &pc, uint64_t a, uint64_t b) {
            const int32_t *key = pc.col[kc];
            for (uint64_t i = a; i < b; i++) mine[hash_key(key[i]) & (P - 1)]++;
        });
#pragma omp barrier
#pragma omp single
        {
            uint64_t acc = 0;
            for (uint32_t p = 0; p < P; p++) {
                off[p] = acc;
                for (int u = 0; u < T; u++) {
                    const uint64_t c = cnt[(size_t)u * P + p];
                    cnt[(size_t)u * P + p] = acc;
                    acc += c;
                }
            }
            off[P] = acc;
        }
        for_range(lo, hi, [&](const Piece &pc, uint64_t a, uint64_t b) {
            const int32_t *key = pc.col[kc];
            for (uint64_t i = a; i < b; i++) {
                const uint64_t pos = mine[hash_key(key[i]) & (P - 1)]++;
                for (int c = 0; c < nc; c++) base[(uint64_t)c * n + pos] = pc.col[c][i];
            }
        });
    }
    for (uint32_t p = 0; p < P; p++) {
        const uint64_t np = off[p + 1] - off[p];
        out->rows[p] = np;
        out->max_rows = std::max(out->max_rows, np);
        if (!np) continue;
        Piece pc;
        for (int c = 0; c < nc; c++) pc.col[c] = base + (uint64_t)c * n + off[p];
        pc.n = np;
        out->part[p].push_back(pc);
    }
    return AMJ_OK;
}

// Smallest power-of-two P with one stage's per-part device memory within
// the budget: probe and build parts twice (double buffer), the build part's
// index (about three times its columns) and the part's result (about twice
// the probe part).
uint32_t parts_for(uint64_t ibytes, uint64_t bbytes, uint64_t budget) {
    const uint64_t need = 4 * ibytes + 5 * bbytes;
    uint64_t p = 1;
    while (p < (1u << 20) && need > budget * p) p <<= 1;
    return (uint32_t)p;
}

// A device relation's columns copied into a pinned block: one piece.
int device_to_host(amj_ctx *ctx, const amj_rel *r, HostTable *t) {
    t->n = r->n;
    if (!r->n) return AMJ_OK;
    Pinned b;
    AMJ_TRY(b.get(ctx, (size_t)r->ncols * r->n * sizeof(int32_t)));
    Piece pc;
    pc.n = r->n;
    for (int c = 0; c < r->ncols; c++) {
        int32_t *dst = b.i32() + (uint64_t)c * r->n;
        AMJ_CUDA_TRY(cudaMemcpyAsync(dst, r->d_cols[c], r->n * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
        pc.col[c] = dst;
    }
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    t->pieces.push_back(pc);
    t->own.push_back(std::move(b));
    return AMJ_OK;
}

// A part result's rows (device columns res.cols[0..nc-1]) grouped on column
// kc into SUB_PARTS groups on the context stream, then copied into one
// pinned block (column c at c * rows, group g's rows contiguous in every
// column, the group counts after the columns) on the second side stream, so
// that the copy overlaps the next part's join.  group_rows_finish waits for
// the copy and hands the groups to the next table.
struct PendingGroup {
    bool active = false;
    Pinned block;
    DBuf<unsigned int> cnt;
    DBuf<int32_t> grouped;
    uint64_t rows = 0;
    int nc = 0;
    cudaEvent_t done = nullptr;
};

int group_rows_start(amj_ctx *ctx, const amj_result &res, int nc, int kc, cudaEvent_t grouped_ev, cudaEvent_t done_ev,
                     PendingGroup *pg) {
    const uint64_t rows = res.rows;
    pg->rows = rows;
    pg->nc = nc;
    pg->done = done_ev;
    AMJ_TRY(pg->block.get(ctx, (size_t)nc * rows * sizeof(int32_t) + SUB_PARTS * sizeof(unsigned int)));
    AMJ_TRY(pg->cnt.alloc(ctx, 2 * SUB_PARTS));   // counts, then cursors
    AMJ_TRY(pg->grouped.alloc(ctx, (size_t)nc * rows));
    AMJ_CUDA_TRY(cudaMemsetAsync(pg->cnt.p, 0, SUB_PARTS * sizeof(unsigned int), ctx->stream));
    const unsigned g = (unsigned)std::min<uint64_t>((rows + 255) / 256, (uint64_t)ctx->num_sms * 8);
    note_launch(ctx);
    sub_count_kernel<<<g, 256, 0, ctx->stream>>>(res.cols[kc], rows, pg->cnt.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_TRY(scan_exclusive_u32(ctx, pg->cnt.p, pg->cnt.p + SUB_PARTS, SUB_PARTS, nullptr));
    SubCols C{};
    for (int c = 0; c < nc; c++) C.src[c] = res.cols[c];
    C.nc = nc;
    C.kc = kc;
    const unsigned gt = (unsigned)std::min<uint64_t>((rows + SUB_TILE - 1) / SUB_TILE, (uint64_t)ctx->num_sms * 8);
    note_launch(ctx);
    sub_scatter_kernel<<<gt, 256, 0, ctx->stream>>>(C, rows, pg->cnt.p + SUB_PARTS, pg->grouped.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_CUDA_TRY(cudaEventRecord(grouped_ev, ctx->stream));
    cudaStream_t back = ctx->side_stream[1];
    AMJ_CUDA_TRY(cudaStreamWaitEvent(back, grouped_ev, 0));
    int32_t *h = pg->block.i32();
    pg->active = true;   // from here the copies may be in flight
    AMJ_CUDA_TRY(cudaMemcpyAsync(h, pg->grouped.p, (size_t)nc * rows * sizeof(int32_t), cudaMemcpyDeviceToHost, back));
    AMJ_CUDA_TRY(cudaMemcpyAsync(h + (uint64_t)nc * rows, pg->cnt.p, SUB_PARTS * sizeof(unsigned int),
                                 cudaMemcpyDeviceToHost, back));
    AMJ_CUDA_TRY(cudaEventRecord(done_ev, back));
    return AMJ_OK;
}

int group_rows_finish(amj_ctx *ctx, PendingGroup *pg, HostTable *T) {
    (void)ctx;
    AMJ_CUDA_TRY(cudaEventSynchronize(pg->done));
    pg->active = false;
    const uint64_t rows = pg->rows;
    const int nc = pg->nc;
    int32_t *h = pg->block.i32();
    const unsigned int *hcnt = reinterpret_cast<const unsigned int *>(h + (uint64_t)nc * rows);
    uint64_t off = 0;
    for (uint32_t s = 0; s < SUB_PARTS; s++) {
        if (hcnt[s]) {
            Piece pc;
            pc.n = hcnt[s];
            for (int c = 0; c < nc; c++) pc.col[c] = h + (uint64_t)c * rows + off;
            T->sub[s].push_back(pc);
            T->pieces.push_back(pc);
        }
        off += hcnt[s];
    }
    if (off != rows) return fail(AMJ_ECUDA, "AMHJ ooc: grouped rows do not add up");
    T->n += rows;
    T->own.push_back(std::move(pg->block));
    pg->grouped.release();   // the copies are done: stream-ordered frees are safe
    pg->cnt.release();
    return AMJ_OK;
}

// X's rows grouped on column kc into SUB_PARTS groups on the device: the
// rows stream through the device in chunks (copied in on the side stream
// while the previous chunk is grouped), and each chunk comes back grouped
// into a pinned block.  Replaces host scattering for tables in host memory.
int group_on_device(amj_ctx *ctx, const HostTable &X, int kc, uint64_t budget, HostTable *out) {
    HostTable T;
    T.attrs = X.attrs;
    T.sub_col = kc;
    T.sub.assign(SUB_PARTS, {});
    const int nc = (int)X.attrs.size();
    if (X.n == 0) {
        *out = std::move(T);
        return AMJ_OK;
    }
    // chunk rows: three chunk buffers within a quarter of the budget
    uint64_t CH = budget / 4 / (3 * (uint64_t)nc * sizeof(int32_t));
    CH = std::max<uint64_t>(1u << 16, std::min<uint64_t>(CH, 1u << 24));
    CH = std::min<uint64_t>(CH, X.n);
    // the chunks as segments of pieces
    struct Seg {
        size_t piece;
        uint64_t lo, hi;
    };
    std::vector<std::vector<Seg>> chunks;
    std::vector<uint64_t> chunk_rows;
    {
        std::vector<Seg> cur;
        uint64_t have = 0;
        for (size_t i = 0; i < X.pieces.size(); i++) {
            uint64_t lo = 0;
            const uint64_t n = X.pieces[i].n;
            while (lo < n) {
                const uint64_t take = std::min(n - lo, CH - have);
                cur.push_back({i, lo, lo + take});
                lo += take;
                have += take;
                if (have == CH) {
                    chunks.push_back(std::move(cur));
                    chunk_rows.push_back(have);
                    cur.clear();
                    have = 0;
                }
            }
        }
        if (have) {
            chunks.push_back(std::move(cur));
            chunk_rows.push_back(have);
        }
    }
    DBuf<int32_t> in[2], grouped;
    DBuf<unsigned int> cnt;
    for (auto &b : in) AMJ_TRY(b.alloc(ctx, (size_t)nc * CH));
    AMJ_TRY(grouped.alloc(ctx, (size_t)nc * CH));
    AMJ_TRY(cnt.alloc(ctx, 2 * SUB_PARTS));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));   // the buffers exist before the side stream writes them
    cudaStream_t up = ctx->side_stream[0];
    struct Events {
        cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};   // [s]: chunk in slot s copied; [2+s]: slot s read
        ~Events() {
            for (auto x : e)
                if (x) (void)cudaEventDestroy(x);
        }
    } ev;
    for (auto &x : ev.e) AMJ_CUDA_TRY(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    auto upload = [&](size_t k, int s) -> int {
        AMJ_CUDA_TRY(cudaStreamWaitEvent(up, ev.e[2 + s], 0));
        uint64_t o = 0;
        for (const Seg &g : chunks[k]) {
            const Piece &pc = X.pieces[g.piece];
            for (int c = 0; c < nc; c++)
                AMJ_CUDA_TRY(cudaMemcpyAsync(in[s].p + (uint64_t)c * CH + o, pc.col[c] + g.lo, (g.hi - g.lo) * 4,
                                             cudaMemcpyHostToDevice, up));
            o += g.hi - g.lo;
        }
        AMJ_CUDA_TRY(cudaEventRecord(ev.e[s], up));
        return AMJ_OK;
    };
    // slot events start out completed
    AMJ_CUDA_TRY(cudaEventRecord(ev.e[2], ctx->stream));
    AMJ_CUDA_TRY(cudaEventRecord(ev.e[3], ctx->stream));
    std::vector<Pinned> blocks(chunks.size());
    int rc = upload(0, 0);
    for (size_t k = 0; k < chunks.size() && rc == AMJ_OK; k++) {
        const int s = (int)(k & 1);
        if (k + 1 < chunks.size()) rc = upload(k + 1, s ^ 1);
        if (rc != AMJ_OK) break;
        const uint64_t rows = chunk_rows[k];
        rc = blocks[k].get(ctx, (size_t)nc * rows * sizeof(int32_t) + SUB_PARTS * sizeof(unsigned int));
        if (rc != AMJ_OK) break;
        cudaError_t e = cudaStreamWaitEvent(ctx->stream, ev.e[s], 0);
        if (e == cudaSuccess) e = cudaMemsetAsync(cnt.p, 0, SUB_PARTS * sizeof(unsigned int), ctx->stream);
        if (e != cudaSuccess) {
            rc = cuda_fail(e, "AMHJ ooc: grouping");
            break;
        }
        const unsigned g = (unsigned)std::min<uint64_t>((rows + 255) / 256, (uint64_t)ctx->num_sms * 8);
        note_launch(ctx);
        sub_count_kernel<<<g, 256, 0, ctx->stream>>>(in[s].p + (uint64_t)kc * CH, rows, cnt.p);
        rc = scan_exclusive_u32(ctx, cnt.p, cnt.p + SUB_PARTS, SUB_PARTS, nullptr);
        if (rc != AMJ_OK) break;
        SubCols C{};
        for (int c = 0; c < nc; c++) C.src[c] = in[s].p + (uint64_t)c * CH;
        C.nc = nc;
        C.kc = kc;
        const unsigned gt = (unsigned)std::min<uint64_t>((rows + SUB_TILE - 1) / SUB_TILE, (uint64_t)ctx->num_sms * 8);
        note_launch(ctx);
        sub_scatter_kernel<<<gt, 256, 0, ctx->stream>>>(C, rows, cnt.p + SUB_PARTS, grouped.p);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(ev.e[2 + s], ctx->stream);   // slot s may be refilled
        int32_t *h = blocks[k].i32();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h, grouped.p, (size_t)nc * rows * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h + (uint64_t)nc * rows, cnt.p, SUB_PARTS * sizeof(unsigned int),
                                cudaMemcpyDeviceToHost, ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "AMHJ ooc: grouping");
    }
    const cudaError_t e1 = cudaStreamSynchronize(up);
    const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    if (rc != AMJ_OK) return rc;
    if (e1 != cudaSuccess) return cuda_fail(e1, "AMHJ ooc: grouping copies");
    if (e2 != cudaSuccess) return cuda_fail(e2, "AMHJ ooc: grouping");
    for (size_t k = 0; k < chunks.size(); k++) {
        const uint64_t rows = chunk_rows[k];
        int32_t *h = blocks[k].i32();
        const unsigned int *hc = reinterpret_cast<const unsigned int *>(h + (uint64_t)nc * rows);
        uint64_t off = 0;
        for (uint32_t g = 0; g < SUB_PARTS; g++) {
            if (hc[g]) {
                Piece pc;
                pc.n = hc[g];
                for (int c = 0; c < nc; c++) pc.col[c] = h + (uint64_t)c * rows + off;
                T.sub[g].push_back(pc);
                T.pieces.push_back(pc);
            }
            off += hc[g];
        }
        if (off != rows) return fail(AMJ_ECUDA, "AMHJ ooc: grouped rows do not add up");
        T.n += rows;
        T.own.push_back(std::move(blocks[k]));
    }
    *out = std::move(T);
    return AMJ_OK;
}

}  // namespace

void pinned_cache_release(amj_ctx *ctx) {
    if (!ctx || !ctx->pinned_cache) return;
    pinned_trim(ctx);
    delete static_cast<PinnedCache *>(ctx->pinned_cache);
    ctx->pinned_cache = nullptr;
}

int amhj_partitioned_execute(amj_ctx *ctx, const HostPlan &hp, int ws, int dro, int flags, amj_result *out) {
    uint64_t budget = ctx->opts.mem_budget;
    if (!budget) {
        size_t fr = 0, tot = 0;
        AMJ_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        budget = fr / 2;
    }
    const bool materialize = (flags & AMJ_F_MATERIALIZE) != 0;
    cudaStream_t up = ctx->side_stream[0];
    struct Events {
        cudaEvent_t e[2] = {nullptr, nullptr};
        ~Events() {
            for (auto x : e)
                if (x) (void)cudaEventDestroy(x);
        }
    } ev;
    for (auto &x : ev.e) AMJ_CUDA_TRY(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    // stage 0's intermediate: the probe relation (host or device columns)
    HostTable I;
    const amj_rel *pr = hp.probe;
    for (int c = 0; c < pr->ncols; c++) I.attrs.push_back(hp.probe_attr[c]);
    if (pr->where == AMJ_MEM_HOST_STREAMED) {
        Piece pc;
        for (int c = 0; c < pr->ncols; c++) pc.col[c] = pr->h_cols[c];
        pc.n = I.n = pr->n;
        if (pc.n) I.pieces.push_back(pc);
    } else {
        AMJ_TRY(device_to_host(ctx, pr, &I));
    }
    uint64_t count = 0, checksum = 0, joins = 0;
    double part_ms = 0, join_ms = 0;   // host clock: partitioning; part copies and joins
    HostTable fin;   // the last stage's rows, when materialised
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
        HostTable Bt;
        for (int c = 0; c < B->ncols; c++) Bt.attrs.push_back((int)B->attrs[c]);
        if (B->where == AMJ_MEM_HOST_STREAMED) {
            Piece pc;
            for (int c = 0; c < B->ncols; c++) pc.col[c] = B->h_cols[c];
            pc.n = Bt.n = B->n;
            if (pc.n) Bt.pieces.push_back(pc);
        } else {
            AMJ_TRY(device_to_host(ctx, B, &Bt));
        }
        const int nci = (int)I.attrs.size(), ncb = B->ncols, ncs = (int)S.size();
        const uint32_t P = parts_for(I.n * 4 * (uint64_t)nci, B->n * 4 * (uint64_t)ncb, budget);
        Parts ip, bp;
        const auto tp0 = std::chrono::steady_clock::now();
        if (P > 1 && P <= SUB_PARTS) {
            // rows not grouped on this key yet go through the device
            if (I.sub_col != ik) AMJ_TRY(group_on_device(ctx, I, ik, budget, &I));
            AMJ_TRY(group_on_device(ctx, Bt, ls.src_col[0], budget, &Bt));
        }
        AMJ_TRY(partition_table(ctx, I, ik, P, &ip));
        AMJ_TRY(partition_table(ctx, Bt, ls.src_col[0], P, &bp));
        const auto tp1 = std::chrono::steady_clock::now();
        part_ms += std::chrono::duration<double, std::milli>(tp1 - tp0).count();
        // device slots for two part pairs
        DBuf<int32_t> dI[2], dB[2];
        for (int s = 0; s < 2; s++) {
            AMJ_TRY(dI[s].alloc(ctx, std::max<uint64_t>(ip.max_rows, 1) * nci));
            AMJ_TRY(dB[s].alloc(ctx, std::max<uint64_t>(bp.max_rows, 1) * ncb));
        }
        AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));   // the slots exist before the side stream writes them
        std::vector<uint32_t> todo;
        for (uint32_t p = 0; p < P; p++)
            if (ip.rows[p] && bp.rows[p]) todo.push_back(p);
        // copy part pair p into slot s on the side stream (columns back to back)
        auto upload = [&](uint32_t p, int s) -> int {
            const uint64_t ni = ip.rows[p], nb = bp.rows[p];
            uint64_t o = 0;
            for (const Piece &pc : ip.part[p]) {
                for (int c = 0; c < nci; c++)
                    AMJ_CUDA_TRY(cudaMemcpyAsync(dI[s].p + (uint64_t)c * ni + o, pc.col[c], pc.n * 4,
                                                 cudaMemcpyHostToDevice, up));
                o += pc.n;
            }
            o = 0;
            for (const Piece &pc : bp.part[p]) {
                for (int c = 0; c < ncb; c++)
                    AMJ_CUDA_TRY(cudaMemcpyAsync(dB[s].p + (uint64_t)c * nb + o, pc.col[c], pc.n * 4,
                                                 cudaMemcpyHostToDevice, up));
                o += pc.n;
            }
            AMJ_CUDA_TRY(cudaEventRecord(ev.e[s], up));
            return AMJ_OK;
        };
        uint32_t pattrs[AMJ_MAX_COLS], battrs[AMJ_MAX_COLS];
        for (int c = 0; c < nci; c++) pattrs[c] = rename(I.attrs[c]);
        for (int c = 0; c < ncb; c++) battrs[c] = rename((int)B->attrs[c]);
        HostTable next;
        next.attrs = S;
        HostTable &dst = last ? fin : next;
        dst.attrs = S;
        // the next stage's key column among this stage's attributes
        const int next_kc =
            last ? -1 : (int)(std::lower_bound(S.begin(), S.end(), hp.lv[j + 1].attr[0]) - S.begin());
        if (!last) {
            next.sub_col = next_kc;
            next.sub.assign(SUB_PARTS, {});
        }
        const int f = (last && !materialize) ? 0 : AMJ_F_MATERIALIZE;   // result columns stay on the device
        PendingGroup pend[2];
        uint32_t npend = 0;
        struct GroupEvents {
            cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};   // [s]: grouped; [2+s]: copied back
            ~GroupEvents() {
                for (auto x : e)
                    if (x) (void)cudaEventDestroy(x);
            }
        } gev;
        for (auto &x : gev.e) AMJ_CUDA_TRY(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
        int rc = todo.empty() ? AMJ_OK : upload(todo[0], 0);
        for (size_t t = 0; t < todo.size() && rc == AMJ_OK; t++) {
            const uint32_t p = todo[t];
            const int s = (int)(t & 1);
            // the other slot's join has returned: fill it with the next pair
            if (t + 1 < todo.size()) rc = upload(todo[t + 1], s ^ 1);
            if (rc != AMJ_OK) break;
            const cudaError_t we = cudaStreamWaitEvent(ctx->stream, ev.e[s], 0);
            if (we != cudaSuccess) {
                rc = cuda_fail(we, "AMHJ ooc: wait for a part copy");
                break;
            }
            const uint64_t ni = ip.rows[p], nb = bp.rows[p];
            const int32_t *pc[AMJ_MAX_COLS], *bc[AMJ_MAX_COLS];
            for (int c = 0; c < nci; c++) pc[c] = dI[s].p + (uint64_t)c * ni;
            for (int c = 0; c < ncb; c++) bc[c] = dB[s].p + (uint64_t)c * nb;
            amj_rel *rp = nullptr, *rb = nullptr;
            rc = amj_rel_create(ctx, ni, nci, pattrs, pc, AMJ_MEM_DEVICE, &rp);
            if (rc == AMJ_OK) rc = amj_rel_create(ctx, nb, ncb, battrs, bc, AMJ_MEM_DEVICE, &rb);
            amj_result res;
            std::memset(&res, 0, sizeof(res));
            amj_rel *pair[2] = {rp, rb};
            if (rc == AMJ_OK) rc = amj_amhj_execute(ctx, AMJ_QUERY_NORMAL, pair, 2, 0, ws, dro, 0, f, &res);
            if (rc == AMJ_OK) {
                joins++;
                if (last) {
                    count += res.count;
                    checksum += res.checksum;
                }
                if (f && res.rows && !last) {
                    // the part's rows grouped by the next key on the device,
                    // then copied into a pinned block of the next table while
                    // the next part is joined (the copy two parts back is
                    // finished first)
                    PendingGroup &pg = pend[npend & 1];
                    if (pg.active) rc = group_rows_finish(ctx, &pg, &dst);
                    if (rc == AMJ_OK)
                        rc = group_rows_start(ctx, res, ncs, next_kc, gev.e[npend & 1], gev.e[2 + (npend & 1)], &pg);
                    npend++;
                } else if (f && res.rows) {
                    // the last stage's rows into a pinned block of the result
                    Pinned b;
                    rc = b.get(ctx, (size_t)ncs * res.rows * sizeof(int32_t));
                    Piece out_pc;
                    out_pc.n = res.rows;
                    for (int a = 0; a < ncs && rc == AMJ_OK; a++) {
                        int32_t *d = b.i32() + (uint64_t)a * res.rows;
                        const cudaError_t e = cudaMemcpyAsync(d, res.cols[a], res.rows * 4, cudaMemcpyDeviceToHost,
                                                              ctx->stream);
                        if (e != cudaSuccess) rc = cuda_fail(e, "AMHJ ooc: part result copy");
                        out_pc.col[a] = d;
                    }
                    if (rc == AMJ_OK) {
                        dst.pieces.push_back(out_pc);
                        dst.own.push_back(std::move(b));
                        dst.n += res.rows;
                    }
                }
                amj_result_release(&res);   // device columns: freed in stream order after the copies
            }
            if (rp) amj_rel_release(rp);
            if (rb) amj_rel_release(rb);
        }
        // the side streams' copies and the result copies end before the
        // partitions and slots go
        const cudaError_t e1 = cudaStreamSynchronize(up);
        const cudaError_t e3 = cudaStreamSynchronize(ctx->side_stream[1]);
        const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
        for (PendingGroup &pg : pend)
            if (pg.active && rc == AMJ_OK && e1 == cudaSuccess && e2 == cudaSuccess && e3 == cudaSuccess)
                rc = group_rows_finish(ctx, &pg, &dst);
        if (e3 != cudaSuccess && rc == AMJ_OK) rc = cuda_fail(e3, "AMHJ ooc: result copies");
        join_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp1).count();
        if (rc != AMJ_OK) return rc;
        if (e1 != cudaSuccess) return cuda_fail(e1, "AMHJ ooc: part copies");
        if (e2 != cudaSuccess) return cuda_fail(e2, "AMHJ ooc: part joins");
        if (!last) I = std::move(next);
    }
    out->count = count;
    out->checksum = checksum;
    out->stats[7] = joins;   // partition pairs joined
    out->kernel_ms[0] = part_ms;
    out->kernel_ms[1] = join_ms;
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
        }
        // the pieces in order, copied on all host cores
        std::vector<uint64_t> at(fin.pieces.size() + 1, 0);
        for (size_t i = 0; i < fin.pieces.size(); i++) at[i + 1] = at[i] + fin.pieces[i].n;
#pragma omp parallel for schedule(dynamic, 1)
        for (long long i = 0; i < (long long)fin.pieces.size(); i++)
            for (int a = 0; a < hp.k; a++)
                std::memcpy(out->cols[a] + at[i], fin.pieces[i].col[a], fin.pieces[i].n * 4);
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
