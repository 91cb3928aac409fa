// orc_gen.cpp - the seeded synthetic inputs, restated for the oracle.
//
// TEST INFRASTRUCTURE ONLY.  The CPU arm of bench.py and the golden-fixture
// script generate their inputs here, so a process that times the reference
// never maps the product library.  The definitions are the ones the product's
// generators document; tests/test_cpu_oracle.py checks both bit for bit.
//
//  * Stream: value i of stream s under seed x is amj_rng_at(x, s, i), a
//    splitmix64 stream jumped to position i (include/amj_checksum.h).
//  * uniform in [lo, hi): lo + floor(r * (hi - lo) / 2^64) (multiply-high).
//  * permutation of 0..n-1: indices sorted by (r_i, i).
//  * Zipf(theta) over ranks 1..D: inverse CDF of the weights k^-theta at
//    u * sum, u the top 53 bits of r_i; the rank r becomes rank_to_key[r].
//  * R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004): level l of edge e draws
//    u = top 53 bits of amj_rng_at(seed, 'RMAT', e * scale + l) and picks
//    quadrant a | b (dst bit) | c (src bit) | d (both); self-loops dropped,
//    every edge oriented (min, max), duplicates removed, and the distinct
//    edges put in the order of mix64(edge ^ mix64(seed ^ 'SHUFF')).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <parallel/algorithm>
#include <utility>
#include <vector>

#include "../include/amj_checksum.h"

namespace {

inline uint64_t mul_hi(uint64_t r, uint64_t range) {
    return (uint64_t)(((unsigned __int128)r * (unsigned __int128)range) >> 64);
}
inline double top53(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace

extern "C" int orc_gen_uniform_i32(int32_t *out, uint64_t n, int64_t lo, int64_t hi_excl, uint64_t seed,
                                   uint64_t stream) {
    if ((!out && n) || hi_excl <= lo || lo < INT32_MIN || hi_excl - 1 > INT32_MAX) return -1;
    const uint64_t range = (uint64_t)(hi_excl - lo);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) out[i] = (int32_t)(lo + (int64_t)mul_hi(amj_rng_at(seed, stream, i), range));
    return 0;
}

extern "C" int orc_gen_permutation_i32(int32_t *out, uint64_t n, uint64_t seed, uint64_t stream) {
    if ((!out && n) || n > (uint64_t)INT32_MAX + 1) return -1;
    std::vector<std::pair<uint64_t, uint32_t>> t(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) t[i] = {amj_rng_at(seed, stream, i), (uint32_t)i};
    __gnu_parallel::sort(t.begin(), t.end());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) out[i] = (int32_t)t[i].second;
    return 0;
}

extern "C" int orc_gen_zipf_i32(int32_t *out, uint64_t n, uint64_t domain, double theta, const int32_t *rank_to_key,
                                uint64_t seed, uint64_t stream) {
    if ((!out && n) || domain == 0 || domain > (uint64_t)INT32_MAX + 1 || !(theta >= 0)) return -1;
    std::vector<double> cdf(domain);
    double sum = 0.0;
    for (uint64_t k = 0; k < domain; k++) cdf[k] = (sum += std::pow((double)(k + 1), -theta));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        const double u = top53(amj_rng_at(seed, stream, i)) * sum;
        uint64_t r = (uint64_t)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
        r = std::min(r, domain - 1);
        out[i] = rank_to_key ? rank_to_key[r] : (int32_t)r;
    }
    return 0;
}

extern "C" int orc_gen_rmat(int scale, uint64_t nedges, double a, double b, double c, uint64_t seed, int32_t *src,
                            int32_t *dst, uint64_t *n_out) {
    if (scale <= 0 || scale > 31 || !src || !dst || !n_out || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return -1;
    const uint64_t none = ~0ull;
    std::vector<uint64_t> e(nedges);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)nedges; i++) {
        uint32_t u = 0, v = 0;
        for (int l = 0; l < scale; l++) {
            const double x = top53(amj_rng_at(seed, 0x524D4154ull, (uint64_t)i * scale + l));
            const uint32_t qu = x >= a + b, qv = (x >= a && x < a + b) || x >= a + b + c;
            u = u << 1 | qu;
            v = v << 1 | qv;
        }
        e[i] = u == v ? none : ((uint64_t)std::min(u, v) << 32 | std::max(u, v));
    }
    __gnu_parallel::sort(e.begin(), e.end());
    uint64_t m = (uint64_t)(std::unique(e.begin(), e.end()) - e.begin());
    if (m && e[m - 1] == none) m--;
    const uint64_t salt = amj_mix64(seed ^ 0x5348554646ull);
    std::vector<std::pair<uint64_t, uint64_t>> t(m);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)m; i++) t[i] = {amj_mix64(e[i] ^ salt), e[i]};
    __gnu_parallel::sort(t.begin(), t.end());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)m; i++) {
        src[i] = (int32_t)(t[i].second >> 32);
        dst[i] = (int32_t)(uint32_t)t[i].second;
    }
    *n_out = m;
    return 0;
}
