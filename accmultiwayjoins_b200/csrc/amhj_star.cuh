// AMHJ flat path for star-shaped count queries.
//
// When every build level is looked up by an attribute of the probe relation
// (a star: a fact table and its dimensions) and compares nothing but that
// key, the levels are independent: a probe row's result is the cross product
// of its matches in each level.  The frontier DFS (amhj_kernel.cuh) visits
// the levels one after another, so the latencies of a row's lookups add up.
// Here one thread takes one probe row, issues the bucket-bound loads of every
// level together, scans each (short) bucket for its key, and counts and
// hashes the product's tuples in attribute order.  A row whose product
// exceeds STAR_MAX_PRODUCT (a skewed dimension) is listed instead and joined
// afterwards by the DFS kernel, which shares such work across warps.
// Count mode only; bucket layout only.  Where the probe columns allow, the
// fact rows reach shared memory by bulk asynchronous copies instead of the
// threads' loads (amhj_star_bulk_kernel).
#pragma once
#include "amhj_probe.cuh"

namespace amj {

constexpr uint32_t STAR_MAX_PRODUCT = 256;

// whether plan P takes the flat path
inline bool star_eligible(const ProbePlan &P) {
    if (P.L < 1 || P.has_inl || P.sort_out || P.fib_level >= 0) return false;
    for (int l = 0; l < P.L; l++) {
        const LevelDesc &lv = P.lv[l];
        if (lv.layout != AMJ_LAYOUT_BUCKET || lv.key_mode != KEY_SINGLE || lv.cmp_mask != 1u) return false;
        bool from_probe = false;
        for (int c = 0; c < P.probe_ncols; c++) from_probe |= P.probe_attr[c] == lv.key_attr[0];
        if (!from_probe) return false;
    }
    return true;
}

// A level's rows in bucket order: key, and column c.  A two-column level
// may carry its (key, payload) pairs interleaved in `slots` (set up for the
// flat path: one 32-byte sector serves both).
__device__ __forceinline__ int32_t star_key(const LevelDesc &lv, uint32_t i) {
    return lv.slots ? lv.slots[i].x : lv.col[0][i];
}
__device__ __forceinline__ int32_t star_col(const LevelDesc &lv, int c, uint32_t i) {
    return lv.slots ? lv.slots[i].y : lv.col[c][i];
}

// One probe row r whose probe columns are in vals: count and hash its
// product of matches, or list it in `over` when the product exceeds
// STAR_MAX_PRODUCT.
__device__ __forceinline__ void star_row(const ProbePlan &P, int32_t *vals, uint64_t r, unsigned long long &cnt,
                                         unsigned long long &chk, uint32_t *over, unsigned int *nover) {
    int32_t key[AMJ_MAX_BUILD_TABLES];
    uint32_t s[AMJ_MAX_BUILD_TABLES], e[AMJ_MAX_BUILD_TABLES];
    // every level's bucket bounds in flight together
#pragma unroll
    for (int l = 0; l < AMJ_MAX_BUILD_TABLES; l++) {
        if (l >= P.L) break;
        key[l] = vals[P.lv[l].key_attr[0]];
        const uint32_t h = (uint32_t)key[l] & P.lv[l].mask;
        s[l] = P.lv[l].buc_ptrs[h];
        e[l] = P.lv[l].buc_ptrs[h + 1];
    }
    uint32_t first[AMJ_MAX_BUILD_TABLES];
    uint64_t prod = 1;
#pragma unroll
    for (int l = 0; l < AMJ_MAX_BUILD_TABLES; l++) {
        if (l >= P.L) break;
        uint32_t nm = 0, f = e[l];
        for (uint32_t i = s[l]; i < e[l]; i++)
            if (star_key(P.lv[l], i) == key[l]) {
                if (nm == 0) f = i;
                nm++;
            }
        first[l] = f;
        prod *= nm;
    }
    if (prod == 0) return;
    if (prod > STAR_MAX_PRODUCT) {
        over[atomicAdd(nover, 1u)] = (uint32_t)(r - P.row_lo);
        return;
    }
    if (prod == 1) {   // unique keys in every level: one tuple
#pragma unroll
        for (int l = 0; l < AMJ_MAX_BUILD_TABLES; l++) {
            if (l >= P.L) break;
            for (int c = 1; c < P.lv[l].ncols; c++) vals[P.lv[l].attr[c]] = star_col(P.lv[l], c, first[l]);
        }
        uint64_t h = AMJ_CHECKSUM_SEED;
        for (int a = 0; a < P.k; a++) h = amj_hash_step(h, vals[a]);
        cnt++;
        chk += h;
        return;
    }
    // the product's tuples: one matching row per level, the last level fastest
    uint32_t pos[AMJ_MAX_BUILD_TABLES];
#pragma unroll
    for (int l = 0; l < AMJ_MAX_BUILD_TABLES; l++)
        if (l < P.L) pos[l] = first[l];
    while (true) {
#pragma unroll
        for (int l = 0; l < AMJ_MAX_BUILD_TABLES; l++) {
            if (l >= P.L) break;
            for (int c = 1; c < P.lv[l].ncols; c++) vals[P.lv[l].attr[c]] = star_col(P.lv[l], c, pos[l]);
        }
        uint64_t h = AMJ_CHECKSUM_SEED;
        for (int a = 0; a < P.k; a++) h = amj_hash_step(h, vals[a]);
        cnt++;
        chk += h;
        // next combination
        int l = P.L - 1;
        for (; l >= 0; l--) {
            uint32_t i = pos[l] + 1;
            while (i < e[l] && star_key(P.lv[l], i) != key[l]) i++;
            if (i < e[l]) {
                pos[l] = i;
                break;
            }
            pos[l] = first[l];
        }
        if (l < 0) break;
    }
}

__device__ __forceinline__ void star_flush(unsigned long long cnt, unsigned long long chk, unsigned long long *count,
                                           unsigned long long *checksum) {
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd(count, cnt);
        atomicAdd(checksum, chk);
    }
}

__global__ __launch_bounds__(256) void amhj_star_kernel(const __grid_constant__ ProbePlan P,
                                                        unsigned long long *count, unsigned long long *checksum,
                                                        uint32_t *over, unsigned int *nover) {
    unsigned long long cnt = 0, chk = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = P.row_lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < P.row_hi; r += stride) {
        int32_t vals[AMJ_MAX_ATTRS];
        for (int c = 0; c < P.probe_ncols; c++) vals[P.probe_attr[c]] = P.probe_col[c][r];
        star_row(P, vals, r, cnt, chk, over, nover);
    }
    star_flush(cnt, chk, count, checksum);
}

// ---- fact rows staged by the copy engine ----
// The same per-row work with the probe rows of a block brought to shared
// memory in batches of STAR_BATCH rows by bulk asynchronous copies
// (cp.async.bulk, one per column; completion counted in bytes on an
// mbarrier), two batches per block in flight: while the block joins batch
// b, batch b + gridDim.x is copied.  Only the copy engine reads the fact
// columns; the threads' own loads are the dimension lookups.  Full batches
// only (the rows after the last full batch are read directly); the host
// checks that every column's first row is 16-byte aligned.  Every wait is
// bounded by P.spin_limit_ns and reports SITE_BULK_COPY when it runs out.
constexpr int STAR_BATCH = 256;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t arrivals) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(arrivals) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// global -> this CTA's shared memory, `bytes` a multiple of 16, both
// addresses 16-byte aligned
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// bounded wait for phase `parity` of bar; false when the limit ran out
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_try_wait(bar, parity))
        if (globaltimer_ns() - t0 > limit_ns) return false;
    return true;
}

__global__ __launch_bounds__(256, 4) void amhj_star_bulk_kernel(const __grid_constant__ ProbePlan P,
                                                             unsigned long long *count,
                                                             unsigned long long *checksum, uint32_t *over,
                                                             unsigned int *nover, DevStatus *status) {
    __shared__ __align__(16) int32_t buf[2][AMJ_MAX_COLS][STAR_BATCH];
    __shared__ __align__(8) uint64_t bar[2];
    const int nc = P.probe_ncols;
    const uint64_t nb = (P.row_hi - P.row_lo) / STAR_BATCH;   // full batches
    const uint32_t bytes = (uint32_t)nc * STAR_BATCH * sizeof(int32_t);
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](uint64_t b, int s) {   // one thread
        mbar_arrive_expect_tx(&bar[s], bytes);
        for (int c = 0; c < nc; c++)
            bulk_copy_g2s(&buf[s][c][0], P.probe_col[c] + P.row_lo + b * STAR_BATCH, STAR_BATCH * sizeof(int32_t),
                          &bar[s]);
    };
    unsigned long long cnt = 0, chk = 0;
    uint32_t parity = 0;   // bit s: the phase buffer s waits for next
    uint64_t b = blockIdx.x;
    if (threadIdx.x == 0 && b < nb) issue(b, 0);
    int s = 0;
    bool failed = false;
    for (; b < nb; b += gridDim.x, s ^= 1) {
        // the next batch into the other buffer, read by everyone before the
        // last barrier
        const uint64_t nxt = b + gridDim.x;
        if (threadIdx.x == 0 && nxt < nb) issue(nxt, s ^ 1);
        const bool ok = mbar_wait_bounded(&bar[s], (parity >> s) & 1u, P.spin_limit_ns);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) report_error(status, (unsigned)-AMJ_ETIMEOUT, SITE_BULK_COPY, b);
            failed = true;
            break;
        }
        parity ^= 1u << s;
        int32_t vals[AMJ_MAX_ATTRS];
        for (int c = 0; c < nc; c++) vals[P.probe_attr[c]] = buf[s][c][threadIdx.x];
        star_row(P, vals, P.row_lo + b * STAR_BATCH + threadIdx.x, cnt, chk, over, nover);
        __syncthreads();
    }
    if (failed) {
        // the other buffer's copy may still be in flight: wait for it (bounded)
        // before the block's shared memory goes
        const uint64_t nxt = b + gridDim.x;
        if (nxt < nb) (void)mbar_wait_bounded(&bar[s ^ 1], (parity >> (s ^ 1)) & 1u, P.spin_limit_ns);
        return;
    }
    // the rows after the last full batch
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = P.row_lo + nb * STAR_BATCH + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < P.row_hi;
         r += stride) {
        int32_t vals[AMJ_MAX_ATTRS];
        for (int c = 0; c < nc; c++) vals[P.probe_attr[c]] = P.probe_col[c][r];
        star_row(P, vals, r, cnt, chk, over, nover);
    }
    star_flush(cnt, chk, count, checksum);
}

// (key, payload) pairs of a two-column level, interleaved
__global__ void star_interleave_kernel(const int32_t *__restrict__ k, const int32_t *__restrict__ v, uint64_t n,
                                       int2 *__restrict__ kv) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        kv[i] = make_int2(k[i], v[i]);
}

// the probe columns of the listed rows (row ids relative to row_lo)
__global__ void star_gather_kernel(const __grid_constant__ ProbePlan P, const uint32_t *rows, uint32_t n,
                                   int32_t *const *out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int c = 0; c < P.probe_ncols; c++) out[c][i] = P.probe_col[c][P.row_lo + rows[i]];
}

}  // namespace amj

namespace amj {

// ---- thread-per-row baseline ----
// The reference's MHJ (MHJ-GPU/Joins/MHJ.cuh:18-122): one thread per probe
// row walks the build levels depth first with backtracking, scanning each
// bucket alone.  Kept as a comparator for the warp-cooperative frontier DFS
// (AMJ_F_THREAD_PER_ROW); bucket layout, count mode.
inline bool thread_row_eligible(const ProbePlan &P) {
    if (P.L < 1 || P.fib_level >= 0) return false;
    for (int l = 0; l < P.L; l++)
        if (P.lv[l].layout != AMJ_LAYOUT_BUCKET) return false;
    return true;
}

__device__ __forceinline__ void thread_row_range(const LevelDesc &lv, const int32_t *vals, uint32_t &s, uint32_t &e) {
    const int32_t k0 = vals[lv.key_attr[0]];
    const uint32_t h = (lv.key_mode == KEY_PAIR ? hash_pair(k0, vals[lv.key_attr[1]]) : (uint32_t)k0) & lv.mask;
    s = lv.buc_ptrs[h];
    e = lv.buc_ptrs[h + 1];
}

__global__ __launch_bounds__(256) void amhj_thread_row_kernel(const __grid_constant__ ProbePlan P,
                                                              unsigned long long *count,
                                                              unsigned long long *checksum) {
    unsigned long long cnt = 0, chk = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = P.row_lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < P.row_hi; r += stride) {
        int32_t vals[AMJ_MAX_ATTRS];
        for (int c = 0; c < P.probe_ncols; c++) vals[P.probe_attr[c]] = P.probe_col[c][r];
        uint32_t pos[AMJ_MAX_BUILD_TABLES], end[AMJ_MAX_BUILD_TABLES];
        int d = 0;
        thread_row_range(P.lv[0], vals, pos[0], end[0]);
        while (true) {
            if (pos[d] >= end[d]) {
                if (d == 0) break;
                d--;
                pos[d]++;
                continue;
            }
            const LevelDesc &lv = P.lv[d];
            const uint32_t i = pos[d];
            bool ok = true;
            for (int c = 0; c < lv.ncols && ok; c++)
                if ((lv.cmp_mask >> c) & 1u) ok = lv.col[c][i] == vals[lv.attr[c]];
            if (!ok) {
                pos[d]++;
                continue;
            }
            for (int c = 0; c < lv.ncols; c++)
                if ((lv.bind_mask >> c) & 1u) vals[lv.attr[c]] = lv.col[c][i];
            if (d == P.L - 1) {
                int32_t t[AMJ_MAX_ATTRS];
                for (int a = 0; a < P.k; a++) t[a] = vals[a];
                if (P.sort_out)   // a degree-ordered copy reports every tuple sorted
                    for (int a = 1; a < P.k; a++)
                        for (int b = a; b > 0 && t[b - 1] > t[b]; b--) {
                            const int32_t x = t[b - 1];
                            t[b - 1] = t[b];
                            t[b] = x;
                        }
                uint64_t h = AMJ_CHECKSUM_SEED;
                for (int a = 0; a < P.k; a++) h = amj_hash_step(h, t[a]);
                cnt++;
                chk += h;
                pos[d]++;
                continue;
            }
            d++;
            thread_row_range(P.lv[d], vals, pos[d], end[d]);
        }
    }
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd(count, cnt);
        atomicAdd(checksum, chk);
    }
}

}  // namespace amj
