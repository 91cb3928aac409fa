/*
 * amj_checksum.h - the order-independent 64-bit result fingerprint shared by
 * the CUDA kernels, the host library and the CPU oracle.
 *
 * A join result is a bag of tuples.  Each tuple is the list of its attribute
 * values in attribute-id order 0..k-1.  Its tuple hash is
 *
 *     h = AMJ_CHECKSUM_SEED
 *     for v in tuple: h = amj_mix64(h ^ (uint32_t)v)
 *
 * and the checksum of the bag is the sum of the tuple hashes modulo 2^64.
 * The sum makes the fingerprint independent of output order (the GPU writes
 * tuples in a nondeterministic order), the chained mix binds every value to
 * its position in the tuple.  amj_mix64 is the splitmix64 finaliser
 * (Steele, Lea, Flood, "Fast splittable pseudorandom number generators",
 * OOPSLA 2014).
 *
 * The reference fingerprints results with an MD5 of a histogram of the low
 * 20 bits of every value (common-utils/res_stat.h:32-133).  That fingerprint
 * is lossy and order-sensitive in its text form; this one replaces it.
 */
#ifndef AMJ_CHECKSUM_H
#define AMJ_CHECKSUM_H

#include <stdint.h>

#if defined(__CUDACC__)
#define AMJ_HD __host__ __device__ __forceinline__
#else
#define AMJ_HD static inline
#endif

#define AMJ_CHECKSUM_SEED 0x9E3779B97F4A7C15ull

AMJ_HD uint64_t amj_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* one step of the tuple hash: fold the next attribute value into h */
AMJ_HD uint64_t amj_hash_step(uint64_t h, int32_t v) {
    return amj_mix64(h ^ (uint64_t)(uint32_t)v);
}

/* hash of a whole tuple given as k values in attribute order */
AMJ_HD uint64_t amj_tuple_hash_k(const int32_t *vals, int k) {
    uint64_t h = AMJ_CHECKSUM_SEED;
    for (int i = 0; i < k; i++) h = amj_hash_step(h, vals[i]);
    return h;
}

/* counter-based random stream used by the seeded generators: value i of
 * stream `stream` under `seed`.  splitmix64 jumped to position i. */
AMJ_HD uint64_t amj_rng_at(uint64_t seed, uint64_t stream, uint64_t i) {
    uint64_t base = amj_mix64(seed ^ (stream * 0xD1B54A32D192ED03ull + 0x8CB92BA72F3D8DD7ull));
    return amj_mix64(base + (i + 1ull) * 0x9E3779B97F4A7C15ull);
}

#endif /* AMJ_CHECKSUM_H */
