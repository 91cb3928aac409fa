// The AMHJ probe kernels.  MODE 0 counts (with the checksum), MODE 1 writes
// (two-pass write or the DRO main pass), MODE 2 is the DRO residual pass.
//
// The pieces are device functions over a plan reference so that one query
// per launch (amhj_probe_kernel, plan in kernel parameter space) and many
// queries per launch (amhj_batch_kernel, each warp holding the plan of its
// current query in shared memory) run the same DFS code.
#pragma once
#include "amhj_probe.cuh"

namespace amj {

enum ProbeMode : int { PM_COUNT = 0, PM_WRITE = 1, PM_RESIDUAL = 2 };

// the device task queue of work sharing and the counters beside it
struct WsQueue {
    ProbeState *st;
    Task *tasks;
    unsigned int *ready;
    DevStatus *status;
};

struct ProbeLaunch {
    ProbePlan P;
    ProbeState *st;
    Task *tasks;
    unsigned int *task_ready;
    Breakpoint *units;
    DevStatus *status;
    uint64_t batch_stride;   // batch b covers rows row_lo + b*batch_stride*32 ...
    uint64_t batch_count;    // number of batches
};

// Work-sharing queue.  Slots are handed out in order by q_tail to pushers and
// by q_head as tickets to idle warps; ticket x takes the task of slot x.
// `busy` counts the warps at work plus the tasks pushed but not yet finished:
// a pusher adds the task's share before publishing it and the warp that takes
// the task inherits it, so busy == 0 means no work is left anywhere.
__device__ __forceinline__ bool ws_push(const ProbePlan &P, const WsQueue &Q, const int32_t *vals, uint32_t s,
                                        uint32_t sz, uint8_t depth, uint16_t qid, uint32_t w) {
    ProbeState *st = Q.st;
    if (ld_volatile_u32(&st->q_tail) >= P.task_cap) return false;
    atomicAdd(&st->busy, 1u);
    const uint32_t slot = atomicAdd(&st->q_tail, 1u);
    if (slot >= P.task_cap) {
        atomicSub(&st->busy, 1u);
        return false;
    }
    Task *t = &Q.tasks[slot];
    for (int a = 0; a < P.k; a++) t->vals[a] = vals[a * 32];
    t->s = s;
    t->aux = 0;
    t->sz = sz;
    t->depth = depth;
    t->m8 = 0;
    t->qid = qid;
    t->w = w;
    __threadfence();
    atomicExch(&Q.ready[slot], 1u);
    atomicAdd(&st->tasks_pushed, 1ull);
    return true;
}

// Split rule shared by every mode so a DRO residual replay truncates exactly
// where the main pass did: a contiguous range longer than twice the task
// size keeps one task's worth; the rest becomes two tasks (pushed only when
// `push` is set).  `vals` points at the entry's column in the frontier.
template <int MODE, bool WS>
__device__ __forceinline__ uint32_t maybe_split(const ProbePlan &P, const WsQueue &Q, const LevelDesc &lv,
                                                const int32_t *vals, uint32_t s, uint32_t sz, int depth,
                                                uint16_t qid, uint32_t w) {
    if (!WS || lv.layout == AMJ_LAYOUT_CUCKOO) return sz;
    const uint32_t chunk = P.task_chunk;
    if (sz <= 2 * chunk) return sz;
    const uint32_t rem = sz - chunk, half = rem / 2;
    if (MODE == PM_RESIDUAL) return chunk;
    // push the tail first so a failure leaves a contiguous kept range
    if (!ws_push(P, Q, vals, s + chunk + half, rem - half, (uint8_t)depth, qid, w)) {
        if (P.dro) report_error(Q.status, (unsigned)-AMJ_EOVERFLOW, SITE_WS_QUEUE, sz);
        return sz;
    }
    if (!ws_push(P, Q, vals, s + chunk, half, (uint8_t)depth, qid, w)) {
        if (P.dro) report_error(Q.status, (unsigned)-AMJ_EOVERFLOW, SITE_WS_QUEUE, sz);
        return chunk + half;
    }
    return chunk;
}

// Idle protocol of work sharing, run by lane 0 of a warp whose own work is
// done.  Returns 1 with a task slot, 0 when all work is done (or on error /
// timeout).  One atomic takes a ticket; the warp then waits for that slot's
// task or for the end of all work, backing off exponentially (64 ns .. 4 us)
// so that waiting warps leave the issue slots to the working ones.
static __device__ int ws_acquire(const WsQueue &Q, uint32_t cap, uint64_t spin_limit_ns, uint32_t &slot_out) {
    ProbeState *st = Q.st;
    __threadfence();
    atomicSub(&st->busy, 1u);
    const uint32_t x = atomicAdd(&st->q_head, 1u);
    const unsigned long long t0 = globaltimer_ns();
    unsigned int backoff = 64;
    while (true) {
        if (x < cap && ld_volatile_u32(&Q.ready[x]) != 0u) {
            __threadfence();
            atomicAdd(&st->tasks_popped, 1ull);
            slot_out = x;
            return 1;
        }
        if (ld_volatile_u32(&st->busy) == 0u) {
            // nothing at work and nothing pending: the ticket's task never comes
            __threadfence();
            if (x < cap && ld_volatile_u32(&Q.ready[x]) != 0u) continue;
            return 0;
        }
        if (ld_volatile_u32(&Q.status->code) != 0u) return 0;
        if (globaltimer_ns() - t0 > spin_limit_ns) {
            report_error(Q.status, (unsigned)-AMJ_ETIMEOUT, SITE_WS_IDLE, x);
            return 0;
        }
        __nanosleep(backoff);
        if (backoff < 4096) backoff <<= 1;
    }
}


// last index r in [0, n) with E[r] <= g (E non-decreasing, E[0] <= g); warp-uniform call
__device__ __forceinline__ uint64_t warp_row_of(const unsigned long long *E, uint64_t n, unsigned long long g, int lane) {
    uint64_t lo = 0, hi = n;   // answer in [lo, hi)
    while (hi - lo > 32) {
        const uint64_t step = (hi - lo + 31) >> 5;
        const uint64_t p = lo + step * (uint64_t)lane;
        const bool le = p < hi && E[p] <= g;
        const int c = __popc(__ballot_sync(AMJ_FULL_MASK, le));   // probes 0..c-1 are <= g, c >= 1
        lo = lo + step * (uint64_t)(c - 1);
        const uint64_t nh = lo + step;
        if (nh < hi) hi = nh;
    }
    const uint64_t p = lo + lane;
    const bool le = p < hi && E[p] <= g;
    return lo + (uint64_t)__popc(__ballot_sync(AMJ_FULL_MASK, le)) - 1;
}

constexpr uint32_t L0_CHUNK = 1024;   // level-0 candidates per work-sharing unit

// A level-0 chunk of the plan's candidate space: candidates [g0, g1) of the
// rows [row, rend).  l0_start holds absolute positions (a batched launch
// shares one prefix array between queries), so the space starts at l0_start[0].
struct L0Chunk {
    unsigned long long g0 = 0, g1 = 0;
    uint64_t row = 0, rend = 0;
};

__device__ __forceinline__ void l0_chunk_setup(const ProbePlan &P, unsigned long long chunk, int lane, L0Chunk &c) {
    const uint64_t rows = P.row_hi - P.row_lo;
    const unsigned long long first = P.l0_start[0], total = P.l0_start[rows];
    c.g0 = first + chunk * (unsigned long long)L0_CHUNK;
    c.g1 = c.g0 + L0_CHUNK < total ? c.g0 + L0_CHUNK : total;
    if (c.g0 < total) {
        c.row = warp_row_of(P.l0_start, rows, c.g0, lane);
        c.rend = warp_row_of(P.l0_start, rows, c.g1 - 1, lane) + 1;
    } else {
        c.row = c.rend = 0;
    }
}

// Depth-0 frontier for rows [rb, re) of a level-0 chunk [g0, g1): lane i
// takes row rb+i with its candidate range clipped to the chunk.
__device__ __forceinline__ void load_l0_group(const ProbePlan &P, char *wbase, unsigned long long g0,
                                              unsigned long long g1, uint64_t rb, uint64_t re, int lane) {
    Frontier F = frontier_at(wbase, P, 0);
    const uint64_t row = rb + lane;
    const bool valid = row < re;
    const uint64_t prow = P.row_lo + row;
    for (int cc = 0; cc < P.probe_ncols; cc++)
        F.vals[P.probe_attr[cc] * 32 + lane] = valid ? P.probe_col[cc][prow] : 0;
    __syncwarp();
    uint32_t s = 0, aux = 0, sz = 0;
    uint8_t m8 = 0;
    if (valid) {
        const unsigned long long e0 = P.l0_start[row], e1 = P.l0_start[row + 1];
        const unsigned long long lo = e0 > g0 ? e0 : g0, hi = e1 < g1 ? e1 : g1;
        if (hi > lo) {
            const uint32_t k0 = (uint32_t)(lo - e0);
            sz = (uint32_t)(hi - lo);
            level_lookup(P.lv[0], [&](int a) { return F.vals[a * 32 + lane]; }, s, aux, m8);
            if (P.lv[0].layout == AMJ_LAYOUT_CUCKOO) {
                uint32_t m = m8;
                for (uint32_t t = 0; t < k0; t++) m &= m - 1;   // drop the first k0 matches
                uint32_t keep = 0;
                for (uint32_t t = 0; t < sz; t++) {
                    const uint32_t low = m & (~m + 1u);
                    keep |= low;
                    m &= m - 1;
                }
                m8 = (uint8_t)keep;
            } else {
                s += k0;
            }
        }
    }
    F.s[lane] = s;
    F.aux[lane] = aux;
    F.m8[lane] = m8;
    F.w[lane] = 1;
    const unsigned long long ps = warp_inclusive_scan((unsigned long long)sz, lane);
    F.psum[lane] = ps;
    if (lane == 31) {
        F.meta[0] = 0;
        F.meta[1] = ps;
        F.meta[2] = 32;
    }
    __syncwarp();
}

// Depth-0 frontier of 32 probe tuples starting at row0, coalesced column loads.
template <int MODE, bool WS>
__device__ __forceinline__ void load_probe_batch(const ProbePlan &P, const WsQueue &Q, char *wbase, uint64_t row0,
                                                 int lane, uint16_t qid) {
    Frontier F = frontier_at(wbase, P, 0);
    const uint64_t row = row0 + lane;
    const bool valid = row < P.row_hi;
    for (int c = 0; c < P.probe_ncols; c++) F.vals[P.probe_attr[c] * 32 + lane] = valid ? P.probe_col[c][row] : 0;
    __syncwarp();
    uint32_t s = 0, aux = 0, sz = 0;
    uint8_t m8 = 0;
    if (valid) {
        sz = level_lookup(P.lv[0], [&](int a) { return F.vals[a * 32 + lane]; }, s, aux, m8);
        sz = maybe_split<MODE, WS>(P, Q, P.lv[0], F.vals + lane, s, sz, 0, qid, 1u);
    }
    F.s[lane] = s;
    F.aux[lane] = aux;
    F.m8[lane] = m8;
    F.w[lane] = 1;
    const unsigned long long ps = warp_inclusive_scan((unsigned long long)sz, lane);
    F.psum[lane] = ps;
    if (lane == 31) {
        F.meta[0] = 0;
        F.meta[1] = ps;
        F.meta[2] = 32;
    }
    __syncwarp();
}

// A work-sharing task becomes the only entry of the frontier at its depth
// (the depths above it are empty).  Returns that depth.
template <int MODE, bool WS>
__device__ __forceinline__ int load_task(const ProbePlan &P, const WsQueue &Q, char *wbase, uint32_t tslot,
                                         int lane) {
    const Task t = Q.tasks[tslot];
    const int td = t.depth;
    for (int d = 0; d < td; d++) {
        Frontier E = frontier_at(wbase, P, d);
        if (lane == 0) {
            E.meta[0] = 0;
            E.meta[1] = 0;
            E.meta[2] = 0;
        }
    }
    Frontier F = frontier_at(wbase, P, td);
    if (lane < P.k) F.vals[lane * 32] = t.vals[lane];
    __syncwarp();
    if (lane == 0) {
        const uint32_t sz = maybe_split<MODE, WS>(P, Q, P.lv[td], F.vals, t.s, t.sz, td, t.qid, t.w);
        F.s[0] = t.s;
        F.aux[0] = t.aux;
        F.m8[0] = t.m8;
        F.w[0] = t.w;
        F.psum[0] = sz;
        F.meta[0] = 0;
        F.meta[1] = sz;
        F.meta[2] = 1;
    }
    __syncwarp();
    return td;
}

// per-warp running totals (lane-local until flushed)
struct ProbeAcc {
    unsigned long long cnt = 0, chk = 0, fib = 0;
};

// output bookkeeping of the unit in progress (direct result output)
struct UnitOut {
    unsigned long long emitted = 0, written = 0, skip = 0;
    bool over = false;
};

// Rows of an inlined filter level that equal the tuple on every column.
template <class Get>
__device__ __forceinline__ uint32_t filter_count(const LevelDesc &fl, Get &&get) {
    uint32_t s, aux;
    uint8_t m8;
    const uint32_t sz = level_lookup(fl, get, s, aux, m8);
    int32_t want[4];
#pragma unroll
    for (int c = 0; c < 4; c++) want[c] = c < fl.ncols ? get(fl.attr[c]) : 0;
    uint32_t m = 0;
    for (uint32_t i = 0; i < sz; i++) {
        int32_t v[4] = {0, 0, 0, 0};
        load_candidate(fl, candidate_slot(fl, s, aux, m8, i), fl.cmp_mask, v);
        bool eq = true;
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < fl.ncols && ((fl.cmp_mask >> c) & 1)) eq &= v[c] == want[c];
        m += eq ? 1u : 0u;
    }
    return m;
}

// Emit this step's tuples: lane tuple tv (hash h) stands for `wt` identical
// tuples (wt = 0: none).  Count mode adds them up; the write modes place them
// at consecutive positions of the output (the residual pass skips the ones
// the main pass wrote).
template <int MODE, bool WT = true>
__device__ __forceinline__ void emit_weighted(const ProbePlan &P, const WsQueue &Q, int lane, const int32_t *tv,
                                              uint64_t h, uint32_t wt, ProbeAcc &acc, UnitOut &u) {
    if (MODE == PM_COUNT) {
        if (!WT) {
            // weights are 0 or 1
            if (wt) {
                acc.cnt++;
                acc.chk += h;
            }
            return;
        }
        acc.cnt += wt;
        acc.chk += (unsigned long long)wt * h;
        return;
    }
    const unsigned long long mine = wt;
    const unsigned long long incl = warp_inclusive_scan(mine, lane);
    const unsigned long long tot = __shfl_sync(AMJ_FULL_MASK, incl, 31);
    if (!tot) return;
    const unsigned long long excl = incl - mine;
    if (MODE == PM_WRITE) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&Q.st->out_cursor, tot);
        base = __shfl_sync(AMJ_FULL_MASK, base, 0);
        acc.cnt += wt;
        acc.chk += (unsigned long long)wt * h;
        for (uint32_t r = 0; r < wt; r++) {
            const unsigned long long pos = base + excl + r;
            if (pos < P.out_cap) {
#pragma unroll
                for (int a = 0; a < AMJ_MAX_ATTRS; a++)
                    if (a < P.k) P.out[a][pos] = tv[a];
            }
        }
        if (!u.over) {
            if (base + tot <= P.out_cap) u.written += tot;
            else {
                u.written += base < P.out_cap ? P.out_cap - base : 0ull;
                u.over = true;
            }
        }
        u.emitted += tot;
        return;
    }
    // residual: this lane's copies are tuples [start, start + wt) of the unit
    const unsigned long long start = u.emitted + excl;
    unsigned long long keep = 0;
    if (wt) keep = start >= u.skip ? wt : (start + wt > u.skip ? start + wt - u.skip : 0ull);
    const unsigned long long kincl = warp_inclusive_scan(keep, lane);
    const unsigned long long ktot = __shfl_sync(AMJ_FULL_MASK, kincl, 31);
    if (ktot) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&Q.st->out_cursor, ktot);
        base = __shfl_sync(AMJ_FULL_MASK, base, 0);
        acc.cnt += keep;
        acc.chk += keep * h;
        for (unsigned long long r = 0; r < keep; r++) {
            const unsigned long long pos = base + (kincl - keep) + r;
            if (pos < P.out_cap) {
#pragma unroll
                for (int a = 0; a < AMJ_MAX_ATTRS; a++)
                    if (a < P.k) P.out[a][pos] = tv[a];
            }
        }
    }
    u.emitted += tot;
}

// Expand one 32-candidate chunk of the frontier at `depth`: compare, run the
// inlined filters that follow the level, then emit (no frontier level left)
// or build the frontier of the next level that is one.
// WT: the plan has inlined filter levels, so entries carry weights; without
// them every level is a frontier depth and every weight is 1.
template <int MODE, bool WS, bool WT>
__device__ __forceinline__ void probe_step(const ProbePlan &P, const WsQueue &Q, uint16_t qid, char *wbase, int lane,
                                           unsigned lt, int &depth, ProbeAcc &acc, UnitOut &u) {
    Frontier F = frontier_at(wbase, P, depth);
    const unsigned long long cursor = F.meta[0], total = F.meta[1];
    const int n = (int)F.meta[2];
    __syncwarp();
    if (cursor >= total) {
        depth = WT ? P.prev_lv[depth] : depth - 1;
        return;
    }
    if (lane == 0) F.meta[0] = cursor + 32;
    const LevelDesc &lv = P.lv[depth];
    const unsigned long long j = cursor + lane;
    bool matched = false, cached = false;
    int o = 0;
    uint32_t cslot = 0;
    int32_t cv[4] = {0, 0, 0, 0};
    if (j < total) {
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (F.psum[mid] > j) hi = mid;
            else lo = mid + 1;
        }
        o = lo;
        const unsigned long long start = o ? F.psum[o - 1] : 0ull;
        if (depth == P.fib_level && (F.m8[o] & FIB_FLAG)) {
            cached = true;
            cslot = F.s[o] + (uint32_t)(j - start);
        } else {
            const uint32_t slot = candidate_slot(lv, F.s[o], F.aux[o], F.m8[o], (uint32_t)(j - start));
            load_candidate(lv, slot, lv.cmp_mask | lv.bind_mask, cv);
            matched = true;
#pragma unroll
            for (int c = 0; c < 4; c++)
                if (c < lv.ncols && ((lv.cmp_mask >> c) & 1)) matched &= (cv[c] == F.vals[lv.attr[c] * 32 + o]);
        }
    }
    if (depth == P.fib_level) {
        // frequent-item buffering: cached suffix tuples are emitted here
        const unsigned cm = __ballot_sync(AMJ_FULL_MASK, cached);
        if (cm) {
            int32_t tv[AMJ_MAX_ATTRS];
            uint64_t h = AMJ_CHECKSUM_SEED;
            uint32_t cw = 0;
            if (cached) {
                cw = WT ? F.w[o] : 1u;
#pragma unroll
                for (int a = 0; a < AMJ_MAX_ATTRS; a++)
                    if (a < P.k) tv[a] = ((P.fib_suffix_attrs >> a) & 1u) ? P.fib_cols[a][cslot] : F.vals[a * 32 + o];
                if (P.sort_out) sort_tuple(tv, P.k);
#pragma unroll
                for (int a = 0; a < AMJ_MAX_ATTRS; a++)
                    if (a < P.k) h = amj_hash_step(h, tv[a]);
                acc.fib += cw;
            }
            emit_weighted<MODE>(P, Q, lane, tv, h, cw, acc, u);
        }
    }
    // the tuple's value of attribute a: this level's bound column, else the frontier
    auto val = [&](int a) -> int32_t {
        const int bc = P.bind_col[depth][a];
        return bc < 0 ? F.vals[a * 32 + o] : (bc == 0 ? cv[0] : bc == 1 ? cv[1] : bc == 2 ? cv[2] : cv[3]);
    };
    const int nd = WT ? (int)P.next_lv[depth] : depth + 1;
    uint32_t wt = matched ? (WT ? F.w[o] : 1u) : 0u;
    if (WT)
        for (int l = depth + 1; l < nd && wt; l++) wt *= filter_count(P.lv[l], val);
    const bool live = wt != 0;
    const unsigned mm = __ballot_sync(AMJ_FULL_MASK, live);
    const int idx = __popc(mm & lt);

    if (nd == P.L) {
        // ---- no frontier level left: emit
        if (!mm) return;
        int32_t tv[AMJ_MAX_ATTRS];
        uint64_t h = AMJ_CHECKSUM_SEED;
        if (live) {
#pragma unroll
            for (int a = 0; a < AMJ_MAX_ATTRS; a++)
                if (a < P.k) tv[a] = val(a);
            if (P.sort_out) sort_tuple(tv, P.k);
#pragma unroll
            for (int a = 0; a < AMJ_MAX_ATTRS; a++)
                if (a < P.k) h = amj_hash_step(h, tv[a]);
        }
        emit_weighted<MODE, WT>(P, Q, lane, tv, h, wt, acc, u);
        return;
    }
    if (!mm) return;

    // ---- live tuples become the frontier of level nd
    Frontier C = frontier_at(wbase, P, nd);
    const LevelDesc &nl = P.lv[nd];
    uint32_t s = 0, aux = 0, sz = 0;
    uint8_t m8 = 0;
    if (live) {
        for (int a = 0; a < P.k; a++) C.vals[a * 32 + idx] = F.vals[a * 32 + o];
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < lv.ncols && ((lv.bind_mask >> c) & 1)) C.vals[lv.attr[c] * 32 + idx] = cv[c];
        int fi = -1;
        if (nd == P.fib_level) fi = fib_find(P, C.vals[nl.key_attr[0] * 32 + idx]);
        if (fi >= 0) {
            s = (uint32_t)P.fib_off[fi];
            sz = (uint32_t)(P.fib_off[fi + 1] - P.fib_off[fi]);
            aux = (uint32_t)fi;
            m8 = FIB_FLAG;
        } else {
            sz = level_lookup(nl, [&](int a) { return C.vals[a * 32 + idx]; }, s, aux, m8);
            sz = maybe_split<MODE, WS>(P, Q, nl, C.vals + idx, s, sz, nd, qid, wt);
        }
        C.s[idx] = s;
        C.aux[idx] = aux;
        C.m8[idx] = m8;
        if (WT) C.w[idx] = wt;
    }
    const unsigned long long ps = warp_inclusive_scan((unsigned long long)(live ? sz : 0u), lane);
    if (live) C.psum[idx] = ps;
    const unsigned long long ctot = __shfl_sync(AMJ_FULL_MASK, ps, 31);
    if (lane == 0) {
        C.meta[0] = 0;
        C.meta[1] = ctot;
        C.meta[2] = (unsigned long long)__popc(mm);
    }
    __syncwarp();
    if (ctot) depth = nd;
}

// level-0 candidate count of probe row i (relative to row_lo) of a plan
__device__ __forceinline__ uint32_t l0_size_of(const ProbePlan &P, uint64_t i) {
    int32_t v[AMJ_MAX_ATTRS];
    for (int c = 0; c < P.probe_ncols; c++) {
        const int a = P.probe_attr[c];
        const int32_t x = P.probe_col[c][P.row_lo + i];
#pragma unroll
        for (int t = 0; t < AMJ_MAX_ATTRS; t++)
            if (t == a) v[t] = x;
    }
    uint32_t s, aux;
    uint8_t m8;
    return level_lookup(P.lv[0], [&](int a) {
        int32_t r = 0;
#pragma unroll
        for (int t = 0; t < AMJ_MAX_ATTRS; t++)
            if (t == a) r = v[t];
        return r;
    }, s, aux, m8);
}

// level-0 candidate counts of probe rows row_lo..row_hi-1
static __global__ void amhj_l0_sizes_kernel(const __grid_constant__ ProbePlan P, unsigned long long *sizes) {
    const uint64_t rows = P.row_hi - P.row_lo;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < rows; i += (uint64_t)gridDim.x * blockDim.x)
        sizes[i] = l0_size_of(P, i);
}

template <int MODE, bool WS, bool WT>
__global__ __launch_bounds__(PROBE_THREADS) void amhj_probe_kernel(const __grid_constant__ ProbeLaunch L) {
    extern __shared__ __align__(16) char smem[];
    const ProbePlan &P = L.P;
    const WsQueue Q{L.st, L.tasks, L.task_ready, L.status};
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    char *wbase = smem + (threadIdx.x >> 5) * P.warp_bytes;
    ProbeAcc acc;
    UnitOut u;
    int depth = -1;

    // unit bookkeeping for direct result output
    uint32_t u_kind = 0, u_id = 0;
    bool u_live = false;
    unsigned long long res_next = 0;   // residual: next breakpoint index
    L0Chunk ch;                        // level-0 chunk in progress

    while (true) {
        if (depth < 0 && ch.row < ch.rend) {
            // ---- next 32 rows of the current level-0 chunk (same unit)
            const uint64_t re = (ch.row + 32 < ch.rend) ? ch.row + 32 : ch.rend;
            load_l0_group(P, wbase, ch.g0, ch.g1, ch.row, re, lane);
            ch.row = re;
            depth = 0;
            continue;
        }
        if (depth < 0) {
            // ---- unit finished: record a breakpoint if its output overflowed
            if (MODE == PM_WRITE && P.dro && u_live && u.over && lane == 0) {
                const unsigned idx = atomicAdd(&L.st->n_units, 1u);
                if (idx < P.unit_cap) {
                    L.units[idx].kind = u_kind;
                    L.units[idx].id = u_id;
                    L.units[idx].written = u.written;
                } else {
                    report_error(L.status, (unsigned)-AMJ_EOVERFLOW, SITE_OUT_OVERFLOW, idx);
                }
            }
            u_live = false;
            u.over = false;
            u.emitted = u.written = 0;

            // ---- acquire the next unit
            int have = 0;          // 1 probe batch, 2 task, 3 level-0 chunk
            uint64_t row0 = 0;
            uint32_t tslot = 0;
            unsigned long long l0c = 0;
            if (MODE == PM_RESIDUAL) {
                if (lane == 0) res_next = atomicAdd(&L.st->next_batch, 1ull);
                res_next = __shfl_sync(AMJ_FULL_MASK, res_next, 0);
                if (res_next >= L.batch_count) break;
                const Breakpoint bp = L.units[res_next];
                u.skip = bp.written;
                if (bp.kind == 0) {
                    have = 1;
                    row0 = P.row_lo + (uint64_t)bp.id * 32;
                } else if (bp.kind == 2) {
                    have = 3;
                    l0c = bp.id;
                } else {
                    have = 2;
                    tslot = bp.id;
                }
            } else {
                unsigned long long b = 0;
                if (lane == 0) b = atomicAdd(&L.st->next_batch, 1ull);
                b = __shfl_sync(AMJ_FULL_MASK, b, 0);
                if (b < L.batch_count) {
                    if (P.lbs) {
                        have = 3;
                        l0c = b;
                        u_kind = 2;
                        u_id = (uint32_t)b;
                    } else {
                        row0 = P.row_lo + b * L.batch_stride * 32;
                        if (row0 < P.row_hi) {
                            have = 1;
                            u_kind = 0;
                            u_id = (uint32_t)(b * L.batch_stride);
                        }
                    }
                }
                if (!have) {
                    if (!WS) break;
                    int got = 0;
                    if (lane == 0) got = ws_acquire(Q, P.task_cap, P.spin_limit_ns, tslot);
                    got = __shfl_sync(AMJ_FULL_MASK, got, 0);
                    tslot = __shfl_sync(AMJ_FULL_MASK, tslot, 0);
                    if (!got) break;
                    have = 2;
                    u_kind = 1;
                    u_id = tslot;
                }
            }
            u_live = true;

            if (have == 3) {
                l0_chunk_setup(P, l0c, lane, ch);
                continue;   // the first group is loaded at the top of the loop
            }
            if (have == 1) {
                load_probe_batch<MODE, WS>(P, Q, wbase, row0, lane, 0);
                depth = 0;
            } else {
                depth = load_task<MODE, WS>(P, Q, wbase, tslot, lane);
            }
            continue;
        }
        probe_step<MODE, WS, WT>(P, Q, 0, wbase, lane, lt, depth, acc, u);
    }

    const unsigned long long cnt = warp_sum(acc.cnt), chk = warp_sum(acc.chk), fib = warp_sum(acc.fib);
    if (lane == 0 && (cnt || chk)) {
        atomicAdd(&L.st->count, cnt);
        atomicAdd(&L.st->checksum, chk);
    }
    if (lane == 0 && fib) atomicAdd(&L.st->fib_rows, fib);
}

// ------------------------------------------------------------- batched --
// Many queries in one persistent launch.  Their level-0 candidate spaces are
// laid end to end (one prefix array over every query's probe rows) and cut
// into L0_CHUNK units; unit_base[q] is the first unit of query q.  A warp
// takes units in order, then work-sharing tasks (which carry their query),
// and keeps the plan of the query it is on in its own shared memory, so a
// switch between queries costs one 1 KB copy.  Counts and checksums go to
// per-query slots.
struct BatchLaunch {
    const ProbePlan *plans;
    const unsigned long long *unit_base;   // nq + 1 entries
    unsigned long long *q_count;
    unsigned long long *q_checksum;
    WsQueue Q;
    uint32_t nq;
    uint32_t task_cap;
    uint64_t spin_limit_ns;
    uint32_t warp_stride;                  // shared bytes per warp: plan copy + frontier
};

constexpr uint32_t BATCH_PLAN_BYTES = (sizeof(ProbePlan) + 15) / 16 * 16;

__device__ __forceinline__ void batch_flush(const BatchLaunch &B, int q, ProbeAcc &acc, int lane) {
    const unsigned long long cnt = warp_sum(acc.cnt), chk = warp_sum(acc.chk);
    if (lane == 0 && q >= 0 && (cnt || chk)) {
        atomicAdd(&B.q_count[q], cnt);
        atomicAdd(&B.q_checksum[q], chk);
    }
    acc.cnt = acc.chk = 0;
}

template <int THREADS, bool WT>
__global__ __launch_bounds__(THREADS) void amhj_batch_kernel(const __grid_constant__ BatchLaunch B) {
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    char *wslot = smem + (threadIdx.x >> 5) * B.warp_stride;
    const ProbePlan &P = *reinterpret_cast<const ProbePlan *>(wslot);
    char *wbase = wslot + BATCH_PLAN_BYTES;
    const unsigned long long total_units = B.unit_base[B.nq];
    ProbeAcc acc;
    UnitOut u;
    L0Chunk ch;
    int depth = -1, cur = -1;

    while (true) {
        if (depth < 0 && ch.row < ch.rend) {
            const uint64_t re = (ch.row + 32 < ch.rend) ? ch.row + 32 : ch.rend;
            load_l0_group(P, wbase, ch.g0, ch.g1, ch.row, re, lane);
            ch.row = re;
            depth = 0;
            continue;
        }
        if (depth < 0) {
            unsigned long long b = 0;
            if (lane == 0) b = atomicAdd(&B.Q.st->next_batch, 1ull);
            b = __shfl_sync(AMJ_FULL_MASK, b, 0);
            int q;
            uint32_t tslot = 0;
            const bool task = b >= total_units;
            if (!task) {
                q = (int)warp_row_of(B.unit_base, B.nq, b, lane);
            } else {
                int got = 0;
                if (lane == 0) got = ws_acquire(B.Q, B.task_cap, B.spin_limit_ns, tslot);
                got = __shfl_sync(AMJ_FULL_MASK, got, 0);
                tslot = __shfl_sync(AMJ_FULL_MASK, tslot, 0);
                if (!got) break;
                q = (int)B.Q.tasks[tslot].qid;
            }
            if (q != cur) {
                batch_flush(B, cur, acc, lane);
                const int4 *src = reinterpret_cast<const int4 *>(B.plans + q);
                int4 *dst = reinterpret_cast<int4 *>(wslot);
                for (uint32_t i = lane; i < sizeof(ProbePlan) / 16; i += 32) dst[i] = src[i];
                __syncwarp();
                cur = q;
            }
            if (!task) {
                l0_chunk_setup(P, b - B.unit_base[q], lane, ch);
            } else {
                depth = load_task<PM_COUNT, true>(P, B.Q, wbase, tslot, lane);
            }
            continue;
        }
        probe_step<PM_COUNT, true, WT>(P, B.Q, (uint16_t)cur, wbase, lane, lt, depth, acc, u);
    }
    batch_flush(B, cur, acc, lane);
}

}  // namespace amj
