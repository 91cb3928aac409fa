// Batched AMHJ: many join queries, one build pass and one persistent probe
// launch, optionally captured once into a CUDA graph and replayed.
//
// The reference runs one query per process (exec_AMHJ.cu:218-246); this
// executor is the batched form of that operator.  Every query is compiled as
// amj_amhj_execute would compile it, then:
//
//  build   all build indexes of all queries at once.  The bucket layout packs
//          every row as (global bucket << 32 | global row), where global
//          bucket = the table's first bucket + its own bucket id, sorts the
//          items once (stable LSD radix sort), gathers the index columns in
//          that order and turns the run lengths into one bucket-offset array.
//          Each table's level descriptor points into the shared arrays.  The
//          open-addressing layout inserts every row into its table's slot
//          range in one kernel.
//  probe   level-0 candidate counts of every query's probe rows, one prefix
//          array over all of them, units of 1024 level-0 candidates per query,
//          and amhj_batch_kernel over the whole unit space plus the shared
//          work-sharing queue.  Counts and checksums land in per-query slots.
//
// Sizes are known on the host once the queries are submitted, so the whole
// device sequence needs no host round trip and can be captured.
#include "amhj_batch.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

namespace amj {

// one build index of the batch
struct BatchJob {
    const int32_t *col[4];
    uint64_t row_base;     // first global row
    uint64_t n;
    uint64_t base;         // first global bucket (bucket layout) or slot (open addressing)
    uint32_t mask;
    int8_t ncols, key_mode, layout, pad;
};

// last j in [0, n) with E[j] <= r (E non-decreasing, E[0] <= r)
__device__ __forceinline__ uint32_t find_last_le(const unsigned long long *E, uint32_t n, unsigned long long r) {
    uint32_t lo = 0, hi = n;   // answer in [lo, hi)
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (E[mid] <= r) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void batch_pack_kernel(const BatchJob *__restrict__ jobs, const unsigned long long *__restrict__ job_rb,
                                  uint32_t njobs, uint64_t rows, uint64_t *__restrict__ items) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
        const BatchJob &J = jobs[find_last_le(job_rb, njobs, r)];
        const uint64_t i = r - J.row_base;
        const int32_t c0 = J.col[0][i];
        const uint32_t key = J.key_mode == KEY_PAIR ? hash_pair(c0, J.col[1][i]) : (uint32_t)c0;
        items[r] = ((J.base + (key & J.mask)) << 32) | (uint32_t)r;
    }
}

__global__ void batch_gather_kernel(const uint64_t *__restrict__ items, uint64_t rows, const BatchJob *__restrict__ jobs,
                                    const unsigned long long *__restrict__ job_rb, uint32_t njobs, int ncols,
                                    int32_t *c0, int32_t *c1, int32_t *c2, int32_t *c3) {
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < rows; p += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)items[p];
        const BatchJob &J = jobs[find_last_le(job_rb, njobs, r)];
        const uint64_t i = r - J.row_base;
        c0[p] = J.col[0][i];
        if (ncols > 1 && J.ncols > 1) c1[p] = J.col[1][i];
        if (ncols > 2 && J.ncols > 2) c2[p] = J.col[2][i];
        if (ncols > 3 && J.ncols > 3) c3[p] = J.col[3][i];
    }
}

// counts[b] += run length of global bucket b (items sorted by bucket)
__global__ void batch_bucket_hist_kernel(const uint64_t *__restrict__ items, uint64_t n, uint32_t *__restrict__ counts) {
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        const uint64_t i = base + lane;
        const bool valid = i < n;
        const uint32_t b = valid ? (uint32_t)(items[i] >> 32) : 0xffffffffu;
        const uint32_t prev = __shfl_up_sync(AMJ_FULL_MASK, b, 1);
        const bool head = valid && (lane == 0 || prev != b);
        const unsigned heads = __ballot_sync(AMJ_FULL_MASK, head);
        const unsigned validm = __ballot_sync(AMJ_FULL_MASK, valid);
        if (head) {
            const unsigned after = heads & ~((2u << lane) - 1u);
            const int end = after ? __ffs(after) - 1 : 32 - __clz(validm);
            atomicAdd(&counts[b], (uint32_t)(end - lane));
        }
    }
}

__global__ void batch_fill_slots_kernel(int2 *slots, uint64_t m) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        slots[i] = make_int2(OA_EMPTY_KEY, 0);
}

// open-addressing insert of rows [row0, row0 + rows) of the job list
__global__ void batch_oa_insert_kernel(const BatchJob *__restrict__ jobs, const unsigned long long *__restrict__ job_rb,
                                       uint32_t njobs, uint64_t row0, uint64_t rows, int2 *slots, DevStatus *st) {
    const unsigned long long empty = ((unsigned long long)0 << 32) | (uint32_t)OA_EMPTY_KEY;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < rows; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = row0 + t;
        const BatchJob &J = jobs[find_last_le(job_rb, njobs, r)];
        const uint64_t i = r - J.row_base;
        const int32_t x = J.col[0][i], y = J.ncols > 1 ? J.col[1][i] : 0;
        if (x == OA_EMPTY_KEY) {
            report_error(st, (unsigned)-AMJ_EINVAL, SITE_OA_FULL, r);
            continue;
        }
        const unsigned long long want = ((unsigned long long)(uint32_t)y << 32) | (uint32_t)x;
        uint32_t s = (J.key_mode == KEY_PAIR ? hash_pair(x, y) : hash_key(x)) & J.mask;
        bool done = false;
        for (uint64_t probe = 0; probe <= J.mask; probe++) {
            const unsigned long long prev = atomicCAS((unsigned long long *)&slots[J.base + s], empty, want);
            if (prev == empty) {
                done = true;
                break;
            }
            s = (s + 1) & J.mask;
        }
        if (!done) report_error(st, (unsigned)-AMJ_EOVERFLOW, SITE_OA_FULL, r);
    }
}

// level-0 candidate counts of every query's probe rows; sizes[rows] = 0
__global__ void batch_l0_sizes_kernel(const ProbePlan *__restrict__ plans, const unsigned long long *__restrict__ qrow,
                                      uint32_t nq, uint64_t rows, unsigned long long *__restrict__ sizes) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r <= rows; r += (uint64_t)gridDim.x * blockDim.x) {
        if (r == rows) {
            sizes[r] = 0;
            continue;
        }
        const uint32_t q = find_last_le(qrow, nq, r);
        sizes[r] = l0_size_of(plans[q], r - qrow[q]);
    }
}

// unit_base[q] = sum over queries before q of ceil(level-0 candidates / L0_CHUNK); one block
__global__ void batch_units_kernel(const unsigned long long *__restrict__ l0, const unsigned long long *__restrict__ qrow,
                                   uint32_t nq, unsigned long long *__restrict__ unit_base) {
    __shared__ unsigned long long wsum[32];
    __shared__ unsigned long long carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t b0 = 0; b0 < nq; b0 += blockDim.x) {
        const uint32_t q = b0 + threadIdx.x;
        unsigned long long u = 0;
        if (q < nq) {
            const unsigned long long c = l0[qrow[q + 1]] - l0[qrow[q]];
            u = (c + L0_CHUNK - 1) / L0_CHUNK;
        }
        const unsigned long long incl = warp_inclusive_scan(u, lane);
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        unsigned long long off = carry;
        for (int w = 0; w < warp; w++) off += wsum[w];
        if (q < nq) unit_base[q] = off + incl - u;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long t = 0;
            for (int w = 0; w < nw; w++) t += wsum[w];
            carry += t;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) unit_base[nq] = carry;
}

__global__ void batch_reset_kernel(ProbeState *st, unsigned int warps) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        st->next_batch = 0;
        st->count = st->checksum = st->out_cursor = st->overflow_rows = 0;
        st->q_head = st->q_tail = 0;
        st->busy = warps;
        st->n_units = 0;
        st->tasks_pushed = st->tasks_popped = 0;
        st->fib_rows = 0;
    }
}

}  // namespace amj

using namespace amj;

struct amj_batch {
    amj_ctx *ctx = nullptr;
    struct Query {
        int qt = 0, flags = 0;
        std::vector<amj_rel *> rels;
        HostPlan hp;
    };
    std::vector<Query> qs;

    // ---- prepared state (valid while `prepared`)
    bool prepared = false;
    amj_batch_opts popts{};
    std::vector<BatchJob> jobs;
    std::vector<unsigned long long> job_rb;
    uint64_t bucket_rows = 0, oa_rows = 0, total_buckets = 0, total_slots = 0, probe_rows = 0;
    int sort_bits = 0, ncols_max = 1;
    uint32_t block = 256, warp_stride = 0;
    bool weighted = false;   // some query has inlined filter levels
    unsigned grid = 0;
    size_t smem = 0;
    DBuf<BatchJob> d_jobs;
    DBuf<unsigned long long> d_job_rb;
    DBuf<uint64_t> items_a, items_b;
    DBuf<int32_t> gcols[4];
    DBuf<uint32_t> gptrs;
    DBuf<int2> gslots;
    DBuf<ProbePlan> plans;
    DBuf<unsigned long long> qrow, sizes, l0, unit_base, q_count, q_checksum;
    DBuf<ProbeState> st;
    DBuf<Task> tasks;
    DBuf<unsigned int> ready;
    uint32_t task_cap = 0;
    unsigned long long launches_per_run = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t done_ev = nullptr;
    cudaStream_t cap_stream = nullptr;
    // pinned host copy of the results: counts[nq], checksums[nq], units, state
    unsigned long long *h_out = nullptr;
    bool replayed = false;

    size_t h_out_bytes = 0;

    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    void unprepare() {
        drop_graph();
        prepared = false;
        jobs.clear();
        job_rb.clear();
        d_jobs.release();
        d_job_rb.release();
        items_a.release();
        items_b.release();
        for (auto &c : gcols) c.release();
        gptrs.release();
        gslots.release();
        plans.release();
        qrow.release();
        sizes.release();
        l0.release();
        unit_base.release();
        q_count.release();
        q_checksum.release();
        st.release();
        tasks.release();
        ready.release();
        if (h_out) cudaFreeHost(h_out);
        h_out = nullptr;
        h_out_bytes = 0;
    }
    // forget the plan but keep every buffer for the next prepare (they only grow)
    void invalidate() {
        drop_graph();
        prepared = false;
        jobs.clear();
        job_rb.clear();
    }
};

namespace amj {

static unsigned batch_grid_for(amj_ctx *ctx, uint64_t n) {
    uint64_t g = (n + 255) / 256, cap = (uint64_t)ctx->num_sms * 16;
    return (unsigned)(g == 0 ? 1 : (g > cap ? cap : g));
}

static uint64_t ctx_task_capacity(const amj_ctx *ctx) { return std::min<uint64_t>(ctx->opts.task_capacity, 0x7fffffffull); }

int normalize_batch_opts(const amj_batch_opts *in, amj_batch_opts *o) {
    std::memset(o, 0, sizeof(*o));
    if (in) *o = *in;
    if (o->layout == 0) o->layout = AMJ_LAYOUT_BUCKET;
    if (o->layout != AMJ_LAYOUT_BUCKET && o->layout != AMJ_LAYOUT_OPEN_ADDR)
        return fail(AMJ_EUNSUPPORTED, "batch: layout must be bucket or open addressing");
    if (o->load_factor < 0.f || o->load_factor > 1.f) return fail(AMJ_EINVAL, "batch: load factor must be in (0, 1]");
    if (o->block_size == 0) o->block_size = 256;
    if (o->block_size != 128 && o->block_size != 256 && o->block_size != 512)
        return fail(AMJ_EINVAL, "batch: block size must be 128, 256 or 512");
    if (o->task_chunk == 0) o->task_chunk = 1024;
    if (o->task_chunk < 32 || o->task_chunk > (1 << 20)) return fail(AMJ_EINVAL, "batch: task chunk out of range");
    if (o->grid_blocks < 0) return fail(AMJ_EINVAL, "batch: negative grid size");
    return AMJ_OK;
}

template <int T, bool WT>
static int batch_kernel_setup(amj_ctx *ctx, size_t smem, unsigned *grid) {
    auto kern = amhj_batch_kernel<T, WT>;
    AMJ_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    AMJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, T, smem));
    if (per_sm < 1) return fail(AMJ_EUNSUPPORTED, "batch: probe frontier does not fit in shared memory");
    *grid = (unsigned)(ctx->num_sms * per_sm);
    return AMJ_OK;
}

// Plan the batch for the given options: jobs, plans, sizes, device buffers.
// grow-only device buffer
template <typename T>
static int ensure(amj_ctx *ctx, DBuf<T> &buf, size_t n) {
    if (buf.p && buf.n >= n) return AMJ_OK;
    buf.release();
    return buf.alloc(ctx, n);
}

static int batch_prepare(amj_batch *b, const amj_batch_opts &o) {
    amj_ctx *ctx = b->ctx;
    b->invalidate();
    const uint32_t nq = (uint32_t)b->qs.size();
    if (nq == 0) return fail(AMJ_EINVAL, "batch: no queries submitted");
    // ---- jobs: one per distinct index; bucket-layout jobs first
    std::map<IndexKey, int> job_of;
    std::vector<std::vector<int>> level_job(nq);
    std::vector<std::vector<const HashIndex *>> level_kept(nq);   // indexes kept by the context's provider
    struct Pending {
        IndexKey key;
        const LevelSpec *ls;
        int layout;
    };
    std::vector<Pending> pend;
    for (uint32_t q = 0; q < nq; q++) {
        const HostPlan &hp = b->qs[q].hp;
        for (int l = 0; l < hp.L; l++) {
            const LevelSpec &ls = hp.lv[l];
            int layout = o.layout;
            if (ls.ncols > 2) layout = AMJ_LAYOUT_BUCKET;   // open addressing holds two columns
            IndexKey key{ls.rel, {-1, -1, -1, -1}, ls.ncols, ls.key_mode, layout};
            for (int c = 0; c < ls.ncols; c++) key.src[c] = ls.src_col[c];
            key.uid = ls.rel->uid;
            key.load_factor = o.load_factor;
            const HashIndex *kept = ctx->iprov ? ctx->iprov->get(ctx, key, ls) : nullptr;
            level_kept[q].push_back(kept);
            if (kept) {
                level_job[q].push_back(-1);
                continue;
            }
            auto it = job_of.find(key);
            if (it == job_of.end()) {
                it = job_of.emplace(key, (int)pend.size()).first;
                pend.push_back({key, &ls, layout});
            }
            level_job[q].push_back(it->second);
        }
    }
    // order: bucket jobs, then open-addressing jobs
    std::vector<int> order(pend.size()), where(pend.size());
    for (size_t i = 0; i < pend.size(); i++) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return (pend[x].layout == AMJ_LAYOUT_BUCKET) > (pend[y].layout == AMJ_LAYOUT_BUCKET);
    });
    const double lf = o.load_factor > 0.f ? o.load_factor : 0.0;
    uint64_t row = 0, bucket = 0, slot = 0;
    b->ncols_max = 1;
    for (size_t t = 0; t < order.size(); t++) {
        const Pending &pd = pend[order[t]];
        where[order[t]] = (int)t;
        const LevelSpec &ls = *pd.ls;
        BatchJob J;
        std::memset(&J, 0, sizeof(J));
        for (int c = 0; c < ls.ncols; c++) J.col[c] = ls.rel->d_cols[ls.src_col[c]];
        J.n = ls.rel->n;
        J.row_base = row;
        J.ncols = (int8_t)ls.ncols;
        J.key_mode = (int8_t)ls.key_mode;
        J.layout = (int8_t)pd.layout;
        if (pd.layout == AMJ_LAYOUT_BUCKET) {
            // the reference's directory is floorPow2(n) buckets; a load factor lf < 1 gives floorPow2(n / lf)
            const uint64_t want = lf > 0.0 ? (uint64_t)((double)J.n / lf) : J.n;
            const uint64_t B = want ? floor_pow2(want) : 1;
            J.base = bucket;
            J.mask = (uint32_t)(B - 1);
            bucket += B;
            b->ncols_max = std::max(b->ncols_max, ls.ncols);
        } else {
            uint64_t cap = ceil_pow2((uint64_t)((double)J.n / (lf > 0.0 ? lf : 0.5)) + 1);
            if (cap < 32) cap = 32;
            J.base = slot;
            J.mask = (uint32_t)(cap - 1);
            slot += cap;
        }
        row += J.n;
        b->jobs.push_back(J);
        b->job_rb.push_back(J.row_base);
    }
    b->total_buckets = bucket;
    b->total_slots = slot;
    b->bucket_rows = 0;
    for (auto &J : b->jobs)
        if (J.layout == AMJ_LAYOUT_BUCKET) b->bucket_rows += J.n;
    b->oa_rows = row - b->bucket_rows;
    if (row >= (1ull << 32)) return fail(AMJ_EUNSUPPORTED, "batch: 2^32 or more build rows in one batch");
    if (bucket >= (1ull << 32) - 1) return fail(AMJ_EUNSUPPORTED, "batch: 2^32 or more buckets in one batch");
    if (slot >= (1ull << 32)) return fail(AMJ_EUNSUPPORTED, "batch: 2^32 or more table slots in one batch");
    int bits = 1;
    while (bits < 32 && (1ull << bits) <= bucket) bits++;
    b->sort_bits = bits;

    // ---- device buffers of the build
    const uint32_t njobs = (uint32_t)b->jobs.size();
    AMJ_TRY(ensure(ctx, b->d_jobs, std::max<uint32_t>(njobs, 1)));
    AMJ_TRY(ensure(ctx, b->d_job_rb, std::max<uint32_t>(njobs, 1)));
    AMJ_CUDA_TRY(cudaMemcpyAsync(b->d_jobs.p, b->jobs.data(), njobs * sizeof(BatchJob), cudaMemcpyHostToDevice,
                                 ctx->stream));
    AMJ_CUDA_TRY(cudaMemcpyAsync(b->d_job_rb.p, b->job_rb.data(), njobs * sizeof(unsigned long long),
                                 cudaMemcpyHostToDevice, ctx->stream));
    const uint64_t br = std::max<uint64_t>(b->bucket_rows, 1);
    AMJ_TRY(ensure(ctx, b->items_a, br));
    AMJ_TRY(ensure(ctx, b->items_b, br));
    for (int c = 0; c < b->ncols_max; c++) AMJ_TRY(ensure(ctx, b->gcols[c], br));
    AMJ_TRY(ensure(ctx, b->gptrs, b->total_buckets + 1));
    if (b->total_slots) AMJ_TRY(ensure(ctx, b->gslots, b->total_slots));

    // ---- plans
    std::vector<unsigned long long> qrow(nq + 1, 0);
    for (uint32_t q = 0; q < nq; q++) qrow[q + 1] = qrow[q] + b->qs[q].hp.probe->n;
    b->probe_rows = qrow[nq];
    AMJ_TRY(ensure(ctx, b->qrow, nq + 1));
    AMJ_TRY(ensure(ctx, b->sizes, b->probe_rows + 1));
    AMJ_TRY(ensure(ctx, b->l0, b->probe_rows + 1));
    AMJ_TRY(ensure(ctx, b->unit_base, nq + 1));
    AMJ_TRY(ensure(ctx, b->q_count, nq));
    AMJ_TRY(ensure(ctx, b->q_checksum, nq));
    AMJ_TRY(ensure(ctx, b->plans, nq));
    AMJ_CUDA_TRY(cudaMemcpyAsync(b->qrow.p, qrow.data(), (nq + 1) * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                                 ctx->stream));
    amj_opts po = ctx->opts;
    po.task_chunk = o.task_chunk;
    std::vector<ProbePlan> hplans(nq);
    uint32_t max_warp_bytes = 0;
    const int32_t *gc[4] = {b->gcols[0].p, b->gcols[1].p, b->gcols[2].p, b->gcols[3].p};
    for (uint32_t q = 0; q < nq; q++) {
        const HostPlan &hp = b->qs[q].hp;
        ProbePlan &P = hplans[q];
        std::memset(&P, 0, sizeof(P));
        plan_common(hp, po, &P);
        P.row_lo = 0;
        P.row_hi = hp.probe->n;
        P.l0_start = b->l0.p + qrow[q];
        P.lbs = 1;
        for (int l = 0; l < hp.L; l++) {
            if (level_kept[q][l]) {
                fill_level_from_index(hp.lv[l], *level_kept[q][l], &P.lv[l]);
                continue;
            }
            const BatchJob &J = b->jobs[where[level_job[q][l]]];
            if (J.layout == AMJ_LAYOUT_BUCKET)
                fill_level_desc(hp.lv[l], J.layout, J.key_mode, J.mask, b->gptrs.p + J.base, gc, nullptr, &P.lv[l]);
            else
                fill_level_desc(hp.lv[l], J.layout, J.key_mode, J.mask, nullptr, gc, b->gslots.p + J.base, &P.lv[l]);
        }
        plan_inline(P);
        max_warp_bytes = std::max(max_warp_bytes, P.warp_bytes);
    }
    AMJ_CUDA_TRY(cudaMemcpyAsync(b->plans.p, hplans.data(), nq * sizeof(ProbePlan), cudaMemcpyHostToDevice,
                                 ctx->stream));
    b->task_cap = hplans[0].task_cap;
    AMJ_TRY(ensure(ctx, b->st, 1));
    AMJ_TRY(ensure(ctx, b->tasks, b->task_cap));
    AMJ_TRY(ensure(ctx, b->ready, b->task_cap));

    // ---- probe launch shape
    b->block = (uint32_t)o.block_size;
    b->warp_stride = (BATCH_PLAN_BYTES + max_warp_bytes + 15) / 16 * 16;
    b->smem = (size_t)(b->block / 32) * b->warp_stride;
    if (b->smem > (size_t)ctx->max_smem_optin) return fail(AMJ_EUNSUPPORTED, "batch: frontier exceeds shared memory");
    b->weighted = false;
    for (const ProbePlan &P : hplans) b->weighted |= P.has_inl != 0;
    if (b->weighted) {
        if (b->block == 128) AMJ_TRY((batch_kernel_setup<128, true>(ctx, b->smem, &b->grid)));
        else if (b->block == 256) AMJ_TRY((batch_kernel_setup<256, true>(ctx, b->smem, &b->grid)));
        else AMJ_TRY((batch_kernel_setup<512, true>(ctx, b->smem, &b->grid)));
    } else {
        if (b->block == 128) AMJ_TRY((batch_kernel_setup<128, false>(ctx, b->smem, &b->grid)));
        else if (b->block == 256) AMJ_TRY((batch_kernel_setup<256, false>(ctx, b->smem, &b->grid)));
        else AMJ_TRY((batch_kernel_setup<512, false>(ctx, b->smem, &b->grid)));
    }
    if (o.grid_blocks > 0 && (unsigned)o.grid_blocks < b->grid) b->grid = (unsigned)o.grid_blocks;
    const size_t hbytes = (2 * (size_t)nq + 1) * sizeof(unsigned long long) + sizeof(ProbeState);
    if (b->h_out_bytes < hbytes) {
        // pinned memory is kept across runs: freeing it synchronises the device
        if (b->h_out) cudaFreeHost(b->h_out);
        b->h_out = nullptr;
        b->h_out_bytes = 0;
        AMJ_CUDA_TRY(cudaMallocHost((void **)&b->h_out, hbytes));
        b->h_out_bytes = hbytes;
    }
    b->popts = o;
    b->prepared = true;
    return AMJ_OK;
}

// timing event; inside a capture it becomes an event-record node of the graph
static int mark(cudaEvent_t e, cudaStream_t s, bool capturing) {
    AMJ_CUDA_TRY(capturing ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal) : cudaEventRecord(e, s));
    return AMJ_OK;
}

// The device sequence of one run (capturable: no host synchronisation).
static int batch_record(amj_batch *b, bool capturing) {
    amj_ctx *ctx = b->ctx;
    cudaStream_t s = ctx->stream;
    const uint32_t nq = (uint32_t)b->qs.size(), njobs = (uint32_t)b->jobs.size();
    const unsigned long long l0 = ctx->launches;
    AMJ_TRY(mark(b->ev[0], s, capturing));
    // ---- build
    if (b->bucket_rows) {
        note_launch(ctx);
        batch_pack_kernel<<<batch_grid_for(ctx, b->bucket_rows), 256, 0, s>>>(b->d_jobs.p, b->d_job_rb.p, njobs,
                                                                              b->bucket_rows, b->items_a.p);
        AMJ_CUDA_TRY(cudaGetLastError());
        uint64_t *sorted = nullptr;
        AMJ_TRY(radix_sort_u64(ctx, b->items_a.p, b->items_b.p, b->bucket_rows, SK_IDENT, 32, 32 + b->sort_bits,
                               &sorted));
        note_launch(ctx);
        batch_gather_kernel<<<batch_grid_for(ctx, b->bucket_rows), 256, 0, s>>>(
            sorted, b->bucket_rows, b->d_jobs.p, b->d_job_rb.p, njobs, b->ncols_max, b->gcols[0].p, b->gcols[1].p,
            b->gcols[2].p, b->gcols[3].p);
        AMJ_CUDA_TRY(cudaGetLastError());
        AMJ_CUDA_TRY(cudaMemsetAsync(b->gptrs.p, 0, (b->total_buckets + 1) * sizeof(uint32_t), s));
        note_launch(ctx);
        batch_bucket_hist_kernel<<<batch_grid_for(ctx, b->bucket_rows), 256, 0, s>>>(sorted, b->bucket_rows,
                                                                                     b->gptrs.p);
        AMJ_CUDA_TRY(cudaGetLastError());
        AMJ_TRY(scan_exclusive_u32(ctx, b->gptrs.p, b->gptrs.p, b->total_buckets + 1, nullptr));
    } else {
        AMJ_CUDA_TRY(cudaMemsetAsync(b->gptrs.p, 0, (b->total_buckets + 1) * sizeof(uint32_t), s));
    }
    if (b->oa_rows) {
        note_launch(ctx);
        batch_fill_slots_kernel<<<batch_grid_for(ctx, b->total_slots), 256, 0, s>>>(b->gslots.p, b->total_slots);
        note_launch(ctx);
        batch_oa_insert_kernel<<<batch_grid_for(ctx, b->oa_rows), 256, 0, s>>>(
            b->d_jobs.p, b->d_job_rb.p, njobs, b->bucket_rows, b->oa_rows, b->gslots.p, ctx->d_status);
        AMJ_CUDA_TRY(cudaGetLastError());
    }
    AMJ_TRY(mark(b->ev[1], s, capturing));
    // ---- probe
    note_launch(ctx);
    batch_l0_sizes_kernel<<<batch_grid_for(ctx, b->probe_rows + 1), 256, 0, s>>>(b->plans.p, b->qrow.p, nq,
                                                                                b->probe_rows, b->sizes.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_TRY(scan_exclusive_u64(ctx, (const uint64_t *)b->sizes.p, (uint64_t *)b->l0.p, b->probe_rows + 1, nullptr));
    note_launch(ctx);
    batch_units_kernel<<<1, 1024, 0, s>>>(b->l0.p, b->qrow.p, nq, b->unit_base.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_CUDA_TRY(cudaMemsetAsync(b->ready.p, 0, (size_t)b->task_cap * sizeof(unsigned int), s));
    AMJ_CUDA_TRY(cudaMemsetAsync(b->q_count.p, 0, nq * sizeof(unsigned long long), s));
    AMJ_CUDA_TRY(cudaMemsetAsync(b->q_checksum.p, 0, nq * sizeof(unsigned long long), s));
    note_launch(ctx);
    batch_reset_kernel<<<1, 32, 0, s>>>(b->st.p, b->grid * (b->block / 32));
    AMJ_CUDA_TRY(cudaGetLastError());
    BatchLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.plans = b->plans.p;
    L.unit_base = b->unit_base.p;
    L.q_count = b->q_count.p;
    L.q_checksum = b->q_checksum.p;
    L.Q = WsQueue{b->st.p, b->tasks.p, b->ready.p, ctx->d_status};
    L.nq = nq;
    L.task_cap = b->task_cap;
    L.spin_limit_ns = (uint64_t)ctx->opts.spin_limit_ms * 1000000ull;
    L.warp_stride = b->warp_stride;
    note_launch(ctx);
    if (b->weighted) {
        if (b->block == 128) amhj_batch_kernel<128, true><<<b->grid, 128, b->smem, s>>>(L);
        else if (b->block == 256) amhj_batch_kernel<256, true><<<b->grid, 256, b->smem, s>>>(L);
        else amhj_batch_kernel<512, true><<<b->grid, 512, b->smem, s>>>(L);
    } else {
        if (b->block == 128) amhj_batch_kernel<128, false><<<b->grid, 128, b->smem, s>>>(L);
        else if (b->block == 256) amhj_batch_kernel<256, false><<<b->grid, 256, b->smem, s>>>(L);
        else amhj_batch_kernel<512, false><<<b->grid, 512, b->smem, s>>>(L);
    }
    AMJ_CUDA_TRY(cudaGetLastError());
    AMJ_TRY(mark(b->ev[2], s, capturing));
    b->launches_per_run = ctx->launches - l0;
    return AMJ_OK;
}

static bool same_opts(const amj_batch_opts &a, const amj_batch_opts &b) {
    return a.layout == b.layout && a.load_factor == b.load_factor && a.block_size == b.block_size &&
           a.task_chunk == b.task_chunk && a.grid_blocks == b.grid_blocks;
}

// Enqueue one run on the context stream: the device sequence (replayed
// graph or eager launches), then the results into pinned host memory and the
// completion event.  Returns without waiting.
int batch_launch(amj_batch *b, const amj_batch_opts &o) {
    amj_ctx *ctx = b->ctx;
    AMJ_CUDA_TRY(cudaSetDevice(ctx->device));
    if (!b->prepared || !same_opts(o, b->popts)) AMJ_TRY(batch_prepare(b, o));
    for (auto &e : b->ev)
        if (!e) AMJ_CUDA_TRY(cudaEventCreate(&e));
    if (!b->done_ev) AMJ_CUDA_TRY(cudaEventCreateWithFlags(&b->done_ev, cudaEventDisableTiming));
    AMJ_TRY(status_reset(ctx));
    b->replayed = false;
    if (o.use_graph) {
        if (!b->exec) {
            // capture on a private stream (the context stream may be the
            // legacy default stream, which cannot capture); only the replay
            // runs on the context stream
            if (!b->cap_stream) AMJ_CUDA_TRY(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
            cudaStream_t user = ctx->stream;
            AMJ_CUDA_TRY(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
            ctx->stream = b->cap_stream;
            const int rc = batch_record(b, true);
            ctx->stream = user;
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(b->cap_stream, &g);
            if (rc != AMJ_OK) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (ce != cudaSuccess) return fail(AMJ_ECUDA, std::string("batch: graph capture: ") + cudaGetErrorString(ce));
            b->graph = g;
            const cudaError_t ie = cudaGraphInstantiate(&b->exec, g, 0);
            if (ie != cudaSuccess) {
                b->drop_graph();
                return fail(AMJ_ECUDA, std::string("batch: graph instantiate: ") + cudaGetErrorString(ie));
            }
        }
        AMJ_CUDA_TRY(cudaGraphLaunch(b->exec, ctx->stream));
        ctx->launches += b->launches_per_run;
        b->replayed = true;
    } else {
        AMJ_TRY(batch_record(b, false));
    }
    const uint32_t nq = (uint32_t)b->qs.size();
    unsigned long long *h = b->h_out;
    AMJ_CUDA_TRY(cudaMemcpyAsync(h, b->q_count.p, nq * 8, cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaMemcpyAsync(h + nq, b->q_checksum.p, nq * 8, cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaMemcpyAsync(h + 2 * nq, b->unit_base.p + nq, 8, cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaMemcpyAsync(h + 2 * nq + 1, b->st.p, sizeof(ProbeState), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaEventRecord(b->done_ev, ctx->stream));
    return AMJ_OK;
}

// drop the submitted queries, keep the buffers for the next ones
void batch_clear(amj_batch *b) {
    b->invalidate();
    b->qs.clear();
}

// whether the last launched run has completed (no waiting)
bool batch_done(amj_batch *b) { return b->done_ev && cudaEventQuery(b->done_ev) == cudaSuccess; }

// Wait for the last launched run and return its results.
int batch_collect(amj_batch *b, uint64_t *counts, uint64_t *checksums, amj_batch_stats *stats) {
    amj_ctx *ctx = b->ctx;
    AMJ_CUDA_TRY(cudaSetDevice(ctx->device));
    AMJ_CUDA_TRY(cudaEventSynchronize(b->done_ev));
    AMJ_TRY(status_check(ctx, "batched AMHJ"));
    const uint32_t nq = (uint32_t)b->qs.size();
    const unsigned long long *h = b->h_out;
    ProbeState hs;
    std::memcpy(&hs, h + 2 * nq + 1, sizeof(hs));
    // a full work-sharing queue only means some ranges were not split: results stay exact
    for (uint32_t q = 0; q < nq; q++) {
        if (counts) counts[q] = h[q];
        if (checksums) checksums[q] = h[nq + q];
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        float ms = 0.f;
        AMJ_CUDA_TRY(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
        stats->build_ms = ms;
        AMJ_CUDA_TRY(cudaEventElapsedTime(&ms, b->ev[1], b->ev[2]));
        stats->probe_ms = ms;
        AMJ_CUDA_TRY(cudaEventElapsedTime(&ms, b->ev[0], b->ev[2]));
        stats->total_ms = ms;
        stats->launches = b->launches_per_run;
        stats->tasks_pushed = hs.tasks_pushed;
        stats->tasks_popped = hs.tasks_popped;
        stats->units = h[2 * nq];
        stats->graph = b->replayed ? 1 : 0;
        stats->build_rows = b->bucket_rows + b->oa_rows;
        stats->build_jobs = b->jobs.size();
    }
    return AMJ_OK;
}

static int batch_run(amj_batch *b, const amj_batch_opts &o, uint64_t *counts, uint64_t *checksums,
                     amj_batch_stats *stats) {
    AMJ_TRY(batch_launch(b, o));
    return batch_collect(b, counts, checksums, stats);
}

// Device bytes a run of these queries allocates, from the relation sizes
// (an upper bound of batch_prepare's buffers plus the sort's scratch).
uint64_t batch_estimate_bytes(const amj_batch *b, const amj_batch_opts &o) {
    const double lf = o.load_factor > 0.f ? o.load_factor : 1.0;
    uint64_t rows = 0, buckets = 0, probe = 0;
    for (const auto &q : b->qs) {
        probe += q.hp.probe->n;
        for (int l = 0; l < q.hp.L; l++) {
            rows += q.hp.lv[l].rel->n;
            buckets += (uint64_t)((double)q.hp.lv[l].rel->n / lf) + 1;
        }
    }
    const uint64_t per_row = 16 + 4 * 4 + 1;   // sort items (2 x 8 B), up to 4 gathered columns, sort counts
    return rows * per_row + buckets * (o.layout == AMJ_LAYOUT_OPEN_ADDR ? 16 : 4) + probe * 16 +
           (uint64_t)b->qs.size() * (sizeof(ProbePlan) + 64) + (uint64_t)(ctx_task_capacity(b->ctx)) * 52 +
           (64ull << 20);
}

}  // namespace amj

extern "C" int amj_batch_create(amj_ctx *ctx, amj_batch **out) {
    if (!ctx || !out) return fail(AMJ_EINVAL, "batch_create: null argument");
    *out = new amj_batch();
    (*out)->ctx = ctx;
    return AMJ_OK;
}

extern "C" int amj_batch_submit(amj_batch *b, int query_type, amj_rel *const *rels, int nrels, int flags,
                                uint32_t *qid) {
    if (!b || !rels || nrels <= 0) return fail(AMJ_EINVAL, "batch_submit: bad arguments");
    if (flags & ~AMJ_F_NO_REORDER) return fail(AMJ_EUNSUPPORTED, "batch_submit: batched queries count only");
    if (b->qs.size() >= 0xffffu) return fail(AMJ_EUNSUPPORTED, "batch_submit: at most 65535 queries per batch");
    for (int i = 0; i < nrels; i++) {
        if (!rels[i]) return fail(AMJ_EINVAL, "batch_submit: null relation");
        if (rels[i]->ctx->device != b->ctx->device)
            return fail(AMJ_EINVAL, "batch_submit: relation on another device");
        if (rels[i]->where == AMJ_MEM_HOST_STREAMED)
            return fail(AMJ_EUNSUPPORTED, "batch_submit: relations must be resident on the device");
    }
    amj_batch::Query q;
    q.qt = query_type;
    q.flags = flags;
    q.rels.assign(rels, rels + nrels);
    AMJ_TRY(compile_plan(query_type, rels, nrels, flags, &q.hp));
    if (q.hp.L == 0) return fail(AMJ_EUNSUPPORTED, "batch_submit: a query needs at least one build relation");
    b->qs.push_back(q);
    b->invalidate();
    if (qid) *qid = (uint32_t)(b->qs.size() - 1);
    return AMJ_OK;
}

extern "C" int amj_batch_run(amj_batch *b, const amj_batch_opts *opts, uint64_t *counts, uint64_t *checksums,
                             amj_batch_stats *stats) {
    if (!b) return fail(AMJ_EINVAL, "batch_run: null batch");
    amj_batch_opts o;
    AMJ_TRY(normalize_batch_opts(opts, &o));
    return batch_run(b, o, counts, checksums, stats);
}

extern "C" int amj_batch_size(const amj_batch *b, uint32_t *queries) {
    if (!b || !queries) return fail(AMJ_EINVAL, "batch_size: null argument");
    *queries = (uint32_t)b->qs.size();
    return AMJ_OK;
}

// Autotuner: every combination of the grid on a sample of the batch (every
// `sample_every`-th query), one untimed and `reps` timed eager runs each,
// best = least median device time.
extern "C" int amj_batch_tune(amj_batch *b, const amj_batch_tune_grid *grid, uint32_t sample_every, int reps,
                              amj_batch_opts *best, double *best_ms) {
    if (!b || !best) return fail(AMJ_EINVAL, "batch_tune: null argument");
    if (b->qs.empty()) return fail(AMJ_EINVAL, "batch_tune: no queries submitted");
    static const float dlf[] = {0.5f, 0.7f, 0.85f};
    static const int dbs[] = {128, 256, 512};
    static const int dtc[] = {32, 64, 128, 256, 512, 1024};
    amj_batch_tune_grid g;
    std::memset(&g, 0, sizeof(g));
    if (grid) g = *grid;
    if (g.n_load_factor == 0) {
        g.n_load_factor = 3;
        for (int i = 0; i < 3; i++) g.load_factor[i] = dlf[i];
    }
    if (g.n_block_size == 0) {
        g.n_block_size = 3;
        for (int i = 0; i < 3; i++) g.block_size[i] = dbs[i];
    }
    if (g.n_task_chunk == 0) {
        g.n_task_chunk = 6;
        for (int i = 0; i < 6; i++) g.task_chunk[i] = dtc[i];
    }
    if (g.n_load_factor > 8 || g.n_block_size > 8 || g.n_task_chunk > 8) return fail(AMJ_EINVAL, "batch_tune: grid too large");
    if (sample_every == 0) sample_every = 1;
    if (reps <= 0) reps = 1;
    amj_batch sub;
    sub.ctx = b->ctx;
    for (size_t q = 0; q < b->qs.size(); q += sample_every) sub.qs.push_back(b->qs[q]);
    double bestv = 1e300;
    amj_batch_opts bo{};
    for (int i = 0; i < g.n_load_factor; i++)
        for (int j = 0; j < g.n_block_size; j++)
            for (int t = 0; t < g.n_task_chunk; t++) {
                amj_batch_opts o{};
                o.layout = g.layout;
                o.load_factor = g.load_factor[i];
                o.block_size = g.block_size[j];
                o.task_chunk = g.task_chunk[t];
                amj_batch_opts n;
                AMJ_TRY(normalize_batch_opts(&o, &n));
                amj_batch_stats st;
                AMJ_TRY(batch_run(&sub, n, nullptr, nullptr, &st));   // warm-up
                std::vector<double> ms;
                for (int r = 0; r < reps; r++) {
                    AMJ_TRY(batch_run(&sub, n, nullptr, nullptr, &st));
                    ms.push_back(st.total_ms);
                }
                std::sort(ms.begin(), ms.end());
                const double med = ms[ms.size() / 2];
                if (med < bestv) {
                    bestv = med;
                    bo = n;
                }
            }
    sub.unprepare();
    for (auto &e : sub.ev)
        if (e) cudaEventDestroy(e);
    bo.use_graph = best->use_graph;
    *best = bo;
    if (best_ms) *best_ms = bestv;
    return AMJ_OK;
}

extern "C" int amj_batch_destroy(amj_batch *b) {
    if (!b) return AMJ_OK;
    if (b->ctx) cudaSetDevice(b->ctx->device);
    b->unprepare();
    for (auto &e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    if (b->done_ev) cudaEventDestroy(b->done_ev);
    delete b;
    return AMJ_OK;
}
