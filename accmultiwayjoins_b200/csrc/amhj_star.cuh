// AMHJ flat paths for star- and chain-shaped queries.
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
// Count mode only; bucket layout only.  Stars and chains in the numbering of
// the reference's benchmarks also have register kernels over 32-byte bucket
// heads (amhj_star_canon_kernel, amhj_chain_canon_kernel, below), and
// materialised stars two flat passes (star_rowcount_kernel,
// star_write_kernel).
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

__global__ __launch_bounds__(256) void amhj_star_kernel(const __grid_constant__ ProbePlan P,
                                                        unsigned long long *count, unsigned long long *checksum,
                                                        uint32_t *over, unsigned int *nover) {
    unsigned long long cnt = 0, chk = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = P.row_lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < P.row_hi; r += stride) {
        int32_t vals[AMJ_MAX_ATTRS];
        for (int c = 0; c < P.probe_ncols; c++) vals[P.probe_attr[c]] = P.probe_col[c][r];
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
                if (P.lv[l].col[0][i] == key[l]) {
                    if (nm == 0) f = i;
                    nm++;
                }
            first[l] = f;
            prod *= nm;
        }
        if (prod == 0) continue;
        if (prod > STAR_MAX_PRODUCT) {
            over[atomicAdd(nover, 1u)] = (uint32_t)(r - P.row_lo);
            continue;
        }
        if (prod == 1) {   // unique keys in every level: one tuple
#pragma unroll
            for (int l = 0; l < AMJ_MAX_BUILD_TABLES; l++) {
                if (l >= P.L) break;
                for (int c = 1; c < P.lv[l].ncols; c++) vals[P.lv[l].attr[c]] = P.lv[l].col[c][first[l]];
            }
            uint64_t h = AMJ_CHECKSUM_SEED;
            for (int a = 0; a < P.k; a++) h = amj_hash_step(h, vals[a]);
            cnt++;
            chk += h;
            continue;
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
                for (int c = 1; c < P.lv[l].ncols; c++) vals[P.lv[l].attr[c]] = P.lv[l].col[c][pos[l]];
            }
            uint64_t h = AMJ_CHECKSUM_SEED;
            for (int a = 0; a < P.k; a++) h = amj_hash_step(h, vals[a]);
            cnt++;
            chk += h;
            // next combination
            int l = P.L - 1;
            for (; l >= 0; l--) {
                uint32_t i = pos[l] + 1;
                while (i < e[l] && P.lv[l].col[0][i] != key[l]) i++;
                if (i < e[l]) {
                    pos[l] = i;
                    break;
                }
                pos[l] = first[l];
            }
            if (l < 0) break;
        }
    }
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd(count, cnt);
        atomicAdd(checksum, chk);
    }
}

// ---- the canonical star, count mode: one 32-byte bucket head a lookup ----
// The shape of the reference's star benchmarks: probe F(0..L-1) and, for
// each key attribute c, one level D_c(c, L + c) of (key, payload) looked up
// by c.  The tuple is then (F's row, the payloads in key order), so every
// index below is a compile-time constant and the row's values stay in
// registers (the general kernel above indexes an attribute array at run time,
// a local-memory array, and loops over the levels).
//
// A probe of random lookups is bound by the L1's tag lookups, one for every
// distinct line a warp's load touches: the general kernel makes four per
// level (two bucket bounds, a key, a payload).  Before the probe every bucket
// of a level gets a 32-byte head, one sector: its bounds and its first
// STAR_HEAD_ROWS rows (key, payload), read by one 256-bit load.  Dimension
// buckets hold one or two rows (keys unique, floorPow2(rows) buckets), so a
// lookup is that one load.  A row whose buckets all hold at most
// STAR_HEAD_ROWS rows, one of them with the key, is one tuple, hashed from
// the keys' shared prefix.  Other rows count their matches per level from
// the bounds and enumerate the product (an odometer over the levels, the
// last fastest); products above STAR_MAX_PRODUCT are listed for the DFS
// kernel as above.
constexpr int STAR_HEAD_ROWS = 3;

struct __align__(32) BucketHead {
    uint32_t s, e;                      // the bucket's rows [s, e)
    int32_t kp[2 * STAR_HEAD_ROWS];     // its first rows' (key, payload), 0 past e
};
static_assert(sizeof(BucketHead) == 32, "a bucket head is one sector");

// A star (star_canon) or chain (chain_canon) plan with its levels in key
// order: star level c is keyed by attribute c, chain level d by d + 1.
struct CanonPlan {
    const int32_t *fact[AMJ_MAX_BUILD_TABLES];     // probe columns (star: attribute c; chain: 0 and 1)
    const BucketHead *head[AMJ_MAX_BUILD_TABLES];  // bucket heads of level c
    const int32_t *key[AMJ_MAX_BUILD_TABLES];      // its key column
    const int32_t *pay[AMJ_MAX_BUILD_TABLES];      // its payload column (star: attribute L + c; chain: c + 2)
    const uint32_t *bp[AMJ_MAX_BUILD_TABLES];      // its bucket starts
    uint32_t nb[AMJ_MAX_BUILD_TABLES];             // its buckets (mask + 1)
    uint32_t mask[AMJ_MAX_BUILD_TABLES];
    uint64_t row_lo, row_hi;
};

// L when star plan P has the canonical shape (filling S but the heads), else 0
inline int star_canon(const ProbePlan &P, CanonPlan &S) {
    const int L = P.L;
    if (L < 1 || 2 * L > AMJ_MAX_ATTRS || P.probe_ncols != L || P.k != 2 * L) return 0;
    for (int c = 0; c < L; c++)
        if (P.probe_attr[c] != c) return 0;
    bool seen[AMJ_MAX_BUILD_TABLES] = {};
    for (int l = 0; l < L; l++) {
        const LevelDesc &lv = P.lv[l];
        const int c = lv.key_attr[0];
        if (c < 0 || c >= L || seen[c] || lv.ncols != 2 || lv.attr[0] != c || lv.attr[1] != L + c) return 0;
        seen[c] = true;
        S.fact[c] = P.probe_col[c];
        S.key[c] = lv.col[0];
        S.pay[c] = lv.col[1];
        S.bp[c] = lv.buc_ptrs;
        S.nb[c] = lv.mask + 1u;
        S.mask[c] = lv.mask;
    }
    S.row_lo = P.row_lo;
    S.row_hi = P.row_hi;
    return L;
}

struct HeadOut {
    BucketHead *p[AMJ_MAX_BUILD_TABLES];
};

// the heads of level blockIdx.y
__global__ void bucket_heads_kernel(const __grid_constant__ CanonPlan S, const __grid_constant__ HeadOut H) {
    const int c = blockIdx.y;
    const uint32_t nb = S.nb[c];
    const uint32_t *bp = S.bp[c];
    for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < nb; h += gridDim.x * blockDim.x) {
        BucketHead o;
        o.s = bp[h];
        o.e = bp[h + 1];
#pragma unroll
        for (int i = 0; i < STAR_HEAD_ROWS; i++) {
            const bool in = o.s + i < o.e;
            o.kp[2 * i] = in ? S.key[c][o.s + i] : 0;
            o.kp[2 * i + 1] = in ? S.pay[c][o.s + i] : 0;
        }
        H.p[c][h] = o;
    }
}

// one 256-bit load of a head (32-byte aligned), through the read-only path
__device__ __forceinline__ void load_head(const BucketHead *p, uint32_t (&w)[8]) {
    asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
        : "l"(p));
}

template <int L>
__global__ __launch_bounds__(256, 4) void amhj_star_canon_kernel(const __grid_constant__ CanonPlan S,
                                                              unsigned long long *count, unsigned long long *checksum,
                                                              uint32_t *over, unsigned int *nover) {
    unsigned long long cnt = 0, chk = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = S.row_lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < S.row_hi; r += stride) {
        int32_t k[L];
#pragma unroll
        for (int c = 0; c < L; c++) k[c] = __ldcs(S.fact[c] + r);
        uint32_t w[L][8];
#pragma unroll
        for (int c = 0; c < L; c++) load_head(S.head[c] + ((uint32_t)k[c] & S.mask[c]), w[c]);
        bool one = true;
        int32_t pay[L];
#pragma unroll
        for (int c = 0; c < L; c++) {
            const uint32_t n = w[c][1] - w[c][0];
            uint32_t nm = 0;
            int32_t p = 0;
#pragma unroll
            for (int i = 0; i < STAR_HEAD_ROWS; i++) {
                const bool m = (uint32_t)i < n && (int32_t)w[c][2 + 2 * i] == k[c];
                nm += m ? 1u : 0u;
                p = m ? (int32_t)w[c][3 + 2 * i] : p;
            }
            one &= (n <= (uint32_t)STAR_HEAD_ROWS) & (nm == 1u);
            pay[c] = p;
        }
        uint64_t hk = AMJ_CHECKSUM_SEED;
#pragma unroll
        for (int c = 0; c < L; c++) hk = amj_hash_step(hk, k[c]);
        if (one) {
            uint64_t h = hk;
#pragma unroll
            for (int c = 0; c < L; c++) h = amj_hash_step(h, pay[c]);
            cnt++;
            chk += h;
            continue;
        }
        uint32_t first[L], e[L];
        uint64_t prod = 1;
#pragma unroll
        for (int c = 0; c < L; c++) {
            e[c] = w[c][1];
            uint32_t nm = 0, f = e[c];
            for (uint32_t i = w[c][0]; i < e[c]; i++)
                if (S.key[c][i] == k[c]) {
                    if (nm == 0) f = i;
                    nm++;
                }
            first[c] = f;
            prod *= nm;
        }
        if (prod == 0) continue;
        if (prod > STAR_MAX_PRODUCT) {
            over[atomicAdd(nover, 1u)] = (uint32_t)(r - S.row_lo);
            continue;
        }
        uint32_t pos[L];
#pragma unroll
        for (int c = 0; c < L; c++) pos[c] = first[c];
        while (true) {
            uint64_t h = hk;
#pragma unroll
            for (int c = 0; c < L; c++) h = amj_hash_step(h, S.pay[c][pos[c]]);
            cnt++;
            chk += h;
            bool carry = true;
#pragma unroll
            for (int c = L - 1; c >= 0; c--) {
                if (carry) {
                    uint32_t i = pos[c] + 1;
                    while (i < e[c] && S.key[c][i] != k[c]) i++;
                    if (i < e[c]) {
                        pos[c] = i;
                        carry = false;
                    } else {
                        pos[c] = first[c];
                    }
                }
            }
            if (carry) break;
        }
    }
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd(count, cnt);
        atomicAdd(checksum, chk);
    }
}

// ---- the canonical chain, count mode: a depth-first walk in registers ----
// The shape of the reference's chain benchmarks: probe R0(0, 1) and levels
// R_d(d + 1, d + 2), level d looked up by the payload of level d - 1 (by
// attribute 1 at d = 0).  One thread walks one probe row's matches depth
// first, each level's lookup one bucket head (its bounds and first rows) and
// the tuple hash extended by one step a level, so a tuple costs one step at
// the last level.  A row whose walk would scan more than CHAIN_ROW_BUDGET
// bucket rows (skewed keys) drops what it counted and is listed for the DFS
// kernel, which shares such work across warps.
constexpr uint32_t CHAIN_ROW_BUDGET = 128;

// L when plan P has the canonical chain shape (filling S but the heads), else 0
inline int chain_canon(const ProbePlan &P, CanonPlan &S) {
    const int L = P.L;
    if (L < 1 || L + 2 > AMJ_MAX_ATTRS || P.probe_ncols != 2 || P.k != L + 2) return 0;
    if (P.has_inl || P.sort_out || P.fib_level >= 0 || P.probe_attr[0] != 0 || P.probe_attr[1] != 1) return 0;
    bool seen[AMJ_MAX_BUILD_TABLES] = {};
    for (int l = 0; l < L; l++) {
        const LevelDesc &lv = P.lv[l];
        const int d = lv.key_attr[0] - 1;
        if (d < 0 || d >= L || seen[d] || lv.layout != AMJ_LAYOUT_BUCKET || lv.key_mode != KEY_SINGLE ||
            lv.cmp_mask != 1u || lv.ncols != 2 || lv.attr[0] != d + 1 || lv.attr[1] != d + 2)
            return 0;
        seen[d] = true;
        S.key[d] = lv.col[0];
        S.pay[d] = lv.col[1];
        S.bp[d] = lv.buc_ptrs;
        S.nb[d] = lv.mask + 1u;
        S.mask[d] = lv.mask;
    }
    S.fact[0] = P.probe_col[0];
    S.fact[1] = P.probe_col[1];
    S.row_lo = P.row_lo;
    S.row_hi = P.row_hi;
    return L;
}

// the matches of key at level D and, through them, the levels below; false
// when the walk ran out of budget
template <int D, int L>
__device__ __forceinline__ bool chain_walk(const CanonPlan &S, int32_t key, uint64_t h, unsigned long long &rc,
                                           unsigned long long &rchk, uint32_t &budget) {
    uint32_t w[8];
    load_head(S.head[D] + ((uint32_t)key & S.mask[D]), w);
    const uint32_t n = w[1] - w[0];
    if (n > budget) return false;
    budget -= n;
    for (uint32_t i = 0; i < n; i++) {
        int32_t k, v;
        if (i < (uint32_t)STAR_HEAD_ROWS) {
            k = (int32_t)(i == 0 ? w[2] : (i == 1 ? w[4] : w[6]));
            v = (int32_t)(i == 0 ? w[3] : (i == 1 ? w[5] : w[7]));
        } else {
            k = S.key[D][w[0] + i];
            v = S.pay[D][w[0] + i];
        }
        if (k != key) continue;
        const uint64_t hv = amj_hash_step(h, v);
        if constexpr (D == L - 1) {
            rc++;
            rchk += hv;
        } else {
            if (!chain_walk<D + 1, L>(S, v, hv, rc, rchk, budget)) return false;
        }
    }
    return true;
}

// four blocks per SM (64 registers) up to three levels; deeper walks keep
// their per-level state in two blocks' worth of registers
template <int L>
__global__ __launch_bounds__(256, L <= 3 ? 4 : 2) void amhj_chain_canon_kernel(const __grid_constant__ CanonPlan S,
                                                               unsigned long long *count, unsigned long long *checksum,
                                                               uint32_t *over, unsigned int *nover) {
    unsigned long long cnt = 0, chk = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = S.row_lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < S.row_hi; r += stride) {
        const int32_t a0 = __ldcs(S.fact[0] + r), a1 = __ldcs(S.fact[1] + r);
        const uint64_t h = amj_hash_step(amj_hash_step(AMJ_CHECKSUM_SEED, a0), a1);
        unsigned long long rc = 0, rchk = 0;
        uint32_t budget = CHAIN_ROW_BUDGET;
        if (chain_walk<0, L>(S, a1, h, rc, rchk, budget)) {
            cnt += rc;
            chk += rchk;
        } else {
            over[atomicAdd(nover, 1u)] = (uint32_t)(r - S.row_lo);
        }
    }
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd(count, cnt);
        atomicAdd(checksum, chk);
    }
}

// ---- materialised star joins (two flat passes) ----
// Pass 1: every probe row's number of result tuples (the product of its
// matches per level).  A scan turns them into output offsets.  Pass 2: every
// row writes its product's tuples from its offset, the last level fastest,
// and adds them to the count and checksum.  A row's tuples are written by
// its own thread, so the pass suits plans whose rows have few matches (the
// 2-relation parts of a staged join, stars over dimensions with unique
// keys); rows are independent, so the result is exact for any product.
__global__ __launch_bounds__(256) void star_rowcount_kernel(const __grid_constant__ ProbePlan P,
                                                            unsigned long long *__restrict__ rc) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = P.row_lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < P.row_hi; r += stride) {
        int32_t vals[AMJ_MAX_ATTRS];
        for (int c = 0; c < P.probe_ncols; c++) vals[P.probe_attr[c]] = P.probe_col[c][r];
        unsigned long long prod = 1;
        for (int l = 0; l < P.L && prod; l++) {
            const int32_t key = vals[P.lv[l].key_attr[0]];
            const uint32_t h = (uint32_t)key & P.lv[l].mask;
            const uint32_t s = P.lv[l].buc_ptrs[h], e = P.lv[l].buc_ptrs[h + 1];
            uint32_t nm = 0;
            for (uint32_t i = s; i < e; i++) nm += P.lv[l].col[0][i] == key;
            prod *= nm;
        }
        rc[r - P.row_lo] = prod;
    }
}

__global__ __launch_bounds__(256) void star_write_kernel(const __grid_constant__ ProbePlan P,
                                                         const unsigned long long *__restrict__ off,
                                                         unsigned long long *count, unsigned long long *checksum) {
    unsigned long long cnt = 0, chk = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = P.row_lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < P.row_hi; r += stride) {
        unsigned long long at = off[r - P.row_lo];
        if (off[r - P.row_lo + 1] == at) continue;   // no tuples
        int32_t vals[AMJ_MAX_ATTRS];
        for (int c = 0; c < P.probe_ncols; c++) vals[P.probe_attr[c]] = P.probe_col[c][r];
        int32_t key[AMJ_MAX_BUILD_TABLES];
        uint32_t first[AMJ_MAX_BUILD_TABLES], pos[AMJ_MAX_BUILD_TABLES], e[AMJ_MAX_BUILD_TABLES];
        for (int l = 0; l < P.L; l++) {
            key[l] = vals[P.lv[l].key_attr[0]];
            const uint32_t h = (uint32_t)key[l] & P.lv[l].mask;
            uint32_t i = P.lv[l].buc_ptrs[h];
            e[l] = P.lv[l].buc_ptrs[h + 1];
            while (P.lv[l].col[0][i] != key[l]) i++;   // a match exists: the row has tuples
            first[l] = pos[l] = i;
        }
        while (true) {
            for (int l = 0; l < P.L; l++)
                for (int c = 1; c < P.lv[l].ncols; c++) vals[P.lv[l].attr[c]] = P.lv[l].col[c][pos[l]];
            uint64_t hsh = AMJ_CHECKSUM_SEED;
            for (int a = 0; a < P.k; a++) {
                hsh = amj_hash_step(hsh, vals[a]);
                P.out[a][at] = vals[a];
            }
            at++;
            cnt++;
            chk += hsh;
            int l = P.L - 1;
            for (; l >= 0; l--) {
                uint32_t i = pos[l] + 1;
                while (i < e[l] && P.lv[l].col[0][i] != key[l]) i++;
                if (i < e[l]) {
                    pos[l] = i;
                    break;
                }
                pos[l] = first[l];
            }
            if (l < 0) break;
        }
    }
    cnt = warp_sum(cnt);
    chk = warp_sum(chk);
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd(count, cnt);
        atomicAdd(checksum, chk);
    }
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
