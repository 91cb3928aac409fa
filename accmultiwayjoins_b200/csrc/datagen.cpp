// Seeded synthetic relations and .db file I/O (host side, OpenMP).
//
// The reference writes its inputs with curand kernels and rand_r
// (MHJ-GPU/uniform_writer_.cu:66, MHJ-GPU/data_generator.cuh:34-54,110-187)
// and reads / writes column-major int32 ".db" files whose name carries the
// schema (common-utils/file_io.h:44-121, MHJ-GPU/QueryProcessor.cuh:41-74).
// Here every generator is a pure function of (seed, stream, index) through a
// counter-based splitmix64 stream, so the same relation is produced on any
// machine and any thread count.  The reference has no R-MAT generator; the
// one below is the standard recursive-quadrant model (Chakrabarti, Zhan,
// Faloutsos, SDM 2004).
#include "amj.h"
#include "amj_checksum.h"
#include "amj_internal.h"

#include <parallel/algorithm>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace {

inline uint64_t bounded(uint64_t r, uint64_t range) {
    return (uint64_t)(((unsigned __int128)r * (unsigned __int128)range) >> 64);
}
inline double unit_double(uint64_t r) { return (double)(r >> 11) * 0x1.0p-53; }

}  // namespace

extern "C" int amj_gen_uniform_i32(int32_t *out, uint64_t n, int64_t lo, int64_t hi_excl,
                                   uint64_t seed, uint64_t stream) {
    if ((!out && n) || hi_excl <= lo) return amj::fail(AMJ_EINVAL, "gen_uniform: bad range");
    if (lo < INT32_MIN || hi_excl - 1 > INT32_MAX) return amj::fail(AMJ_EINVAL, "gen_uniform: range exceeds int32");
    const uint64_t range = (uint64_t)(hi_excl - lo);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++)
        out[i] = (int32_t)(lo + (int64_t)bounded(amj_rng_at(seed, stream, (uint64_t)i), range));
    return AMJ_OK;
}

// A uniformly random permutation of 0..n-1: sort indices by a random 64-bit
// tag (ties broken by index).  Deterministic for a given (seed, stream).
extern "C" int amj_gen_permutation_i32(int32_t *out, uint64_t n, uint64_t seed, uint64_t stream) {
    if ((!out && n) || n > (uint64_t)INT32_MAX + 1) return amj::fail(AMJ_EINVAL, "gen_permutation: bad n");
    std::vector<std::pair<uint64_t, uint32_t>> tag(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) tag[i] = {amj_rng_at(seed, stream, (uint64_t)i), (uint32_t)i};
    __gnu_parallel::sort(tag.begin(), tag.end());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) out[i] = (int32_t)tag[i].second;
    return AMJ_OK;
}

// Zipf(theta) over ranks 1..domain by inverse CDF of weights 1/k^theta; the
// drawn rank r (0-based) becomes rank_to_key[r] when a mapping is given, so a
// caller can scatter the frequent ranks over the key domain the way the
// reference permutes ranks (MHJ-GPU/data_generator.cuh:149-162).
extern "C" int amj_gen_zipf_i32(int32_t *out, uint64_t n, uint64_t domain, double theta,
                                const int32_t *rank_to_key, uint64_t seed, uint64_t stream) {
    if ((!out && n) || domain == 0 || domain > (uint64_t)INT32_MAX + 1 || !(theta >= 0))
        return amj::fail(AMJ_EINVAL, "gen_zipf: bad arguments");
    std::vector<double> cdf(domain);
    double acc = 0.0;
    for (uint64_t k = 0; k < domain; k++) {
        acc += std::pow((double)(k + 1), -theta);
        cdf[k] = acc;
    }
    const double total = acc;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        double u = unit_double(amj_rng_at(seed, stream, (uint64_t)i)) * total;
        uint64_t r = (uint64_t)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
        if (r >= domain) r = domain - 1;
        out[i] = rank_to_key ? rank_to_key[r] : (int32_t)r;
    }
    return AMJ_OK;
}

extern "C" int amj_gen_rmat(int scale, uint64_t nedges, double a, double b, double c, uint64_t seed,
                            int32_t *src, int32_t *dst, uint64_t *n_out) {
    if (scale <= 0 || scale > 31 || !src || !dst || !n_out || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
        return amj::fail(AMJ_EINVAL, "gen_rmat: bad arguments");
    const double ab = a + b, abc = a + b + c;
    std::vector<uint64_t> keys(nedges);
    // draw: level l picks bit (scale-1-l) of source and destination
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)nedges; e++) {
        uint32_t u = 0, v = 0;
        for (int l = 0; l < scale; l++) {
            double x = unit_double(amj_rng_at(seed, 0x524D4154ull, (uint64_t)e * (uint64_t)scale + (uint64_t)l));
            uint32_t bu = 0, bv = 0;
            if (x < a) {
            } else if (x < ab) {
                bv = 1;
            } else if (x < abc) {
                bu = 1;
            } else {
                bu = 1;
                bv = 1;
            }
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        // orient u<v; a self-loop becomes an all-ones sentinel that sorts last
        if (u == v) keys[e] = ~0ull;
        else {
            uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
            keys[e] = ((uint64_t)lo << 32) | hi;
        }
    }
    __gnu_parallel::sort(keys.begin(), keys.end());
    uint64_t m = (uint64_t)(std::unique(keys.begin(), keys.end()) - keys.begin());
    if (m && keys[m - 1] == ~0ull) m--;
    // shuffle the distinct edges so the relation is not presorted
    std::vector<std::pair<uint64_t, uint64_t>> tagged(m);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)m; i++)
        tagged[i] = {amj_mix64(keys[i] ^ amj_mix64(seed ^ 0x5348554646ull)), keys[i]};
    __gnu_parallel::sort(tagged.begin(), tagged.end());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)m; i++) {
        src[i] = (int32_t)(tagged[i].second >> 32);
        dst[i] = (int32_t)(tagged[i].second & 0xffffffffu);
    }
    *n_out = m;
    return AMJ_OK;
}

extern "C" int amj_checksum_host(const int32_t *const *cols, int k, uint64_t n, uint64_t *out) {
    if (!out || k < 0 || k > AMJ_MAX_ATTRS || (n && !cols)) return amj::fail(AMJ_EINVAL, "checksum_host: bad arguments");
    uint64_t total = 0;
#pragma omp parallel for reduction(+ : total) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        uint64_t h = AMJ_CHECKSUM_SEED;
        for (int a = 0; a < k; a++) h = amj_hash_step(h, cols[a][i]);
        total += h;
    }
    *out = total;
    return AMJ_OK;
}

// ---- .db files ----

extern "C" int amj_db_parse_name(const char *path, uint64_t *n, int *ncols, uint32_t *attrs) {
    if (!path) return amj::fail(AMJ_EINVAL, "db_parse_name: null path");
    std::string p(path);
    size_t slash = p.find_last_of('/');
    std::string base = slash == std::string::npos ? p : p.substr(slash + 1);
    if (base.size() < 4 || base.compare(base.size() - 3, 3, ".db") != 0)
        return amj::fail(AMJ_EINVAL, "db_parse_name: not a .db file: " + base);
    base = base.substr(0, base.size() - 3);
    std::vector<std::string> parts;
    size_t s = 0;
    while (true) {
        size_t u = base.find('_', s);
        parts.push_back(base.substr(s, u == std::string::npos ? std::string::npos : u - s));
        if (u == std::string::npos) break;
        s = u + 1;
    }
    if (parts.size() < 2 || parts.size() - 1 > AMJ_MAX_COLS)
        return amj::fail(AMJ_EINVAL, "db_parse_name: expected <rows>_<attr>..: " + base);
    try {
        uint64_t rows = std::stoull(parts[0]);
        if (n) *n = rows;
        if (ncols) *ncols = (int)parts.size() - 1;
        for (size_t i = 1; i < parts.size(); i++) {
            unsigned long v = std::stoul(parts[i]);
            if (v >= AMJ_MAX_ATTRS) return amj::fail(AMJ_EINVAL, "db_parse_name: attribute id too large");
            if (attrs) attrs[i - 1] = (uint32_t)v;
        }
    } catch (...) {
        return amj::fail(AMJ_EINVAL, "db_parse_name: non-numeric field in " + base);
    }
    return AMJ_OK;
}

extern "C" int amj_db_write(const char *path, uint64_t n, int ncols, const int32_t *const *cols) {
    if (!path || ncols <= 0 || ncols > AMJ_MAX_COLS || (n && !cols)) return amj::fail(AMJ_EINVAL, "db_write: bad arguments");
    FILE *f = std::fopen(path, "wb");
    if (!f) return amj::fail(AMJ_EIO, std::string("db_write: cannot open ") + path);
    for (int c = 0; c < ncols; c++) {
        if (n && std::fwrite(cols[c], sizeof(int32_t), n, f) != n) {
            std::fclose(f);
            return amj::fail(AMJ_EIO, std::string("db_write: short write to ") + path);
        }
    }
    if (std::fclose(f) != 0) return amj::fail(AMJ_EIO, std::string("db_write: close failed for ") + path);
    return AMJ_OK;
}

extern "C" int amj_db_read(const char *path, uint64_t n, int ncols, int32_t *const *cols) {
    if (!path || ncols <= 0 || ncols > AMJ_MAX_COLS || (n && !cols)) return amj::fail(AMJ_EINVAL, "db_read: bad arguments");
    int fd = ::open(path, O_RDONLY);
    if (fd < 0) return amj::fail(AMJ_EIO, std::string("db_read: cannot open ") + path);
    struct stat st;
    if (fstat(fd, &st) != 0) {
        ::close(fd);
        return amj::fail(AMJ_EIO, std::string("db_read: stat failed for ") + path);
    }
    const uint64_t need = n * (uint64_t)ncols * sizeof(int32_t);
    if ((uint64_t)st.st_size != need) {
        ::close(fd);
        return amj::fail(AMJ_EIO, std::string("db_read: size mismatch (file holds ") + std::to_string(st.st_size) +
                                      " bytes, schema needs " + std::to_string(need) + ") in " + path);
    }
    if (need == 0) {
        ::close(fd);
        return AMJ_OK;
    }
    void *m = mmap(nullptr, need, PROT_READ, MAP_PRIVATE, fd, 0);
    ::close(fd);
    if (m == MAP_FAILED) return amj::fail(AMJ_EIO, std::string("db_read: mmap failed for ") + path);
    const int32_t *src = (const int32_t *)m;
    for (int c = 0; c < ncols; c++) std::memcpy(cols[c], src + (uint64_t)c * n, n * sizeof(int32_t));
    munmap(m, need);
    return AMJ_OK;
}
