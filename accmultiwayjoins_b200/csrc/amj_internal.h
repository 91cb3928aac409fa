// Host-side internals shared by every translation unit of libamj: the
// thread-local error message and the status helpers.
#pragma once
#include <string>
#include "amj.h"

namespace amj {

// Record `msg` as the calling thread's last error and return `code`.
int fail(int code, const std::string &msg);

inline uint64_t floor_pow2(uint64_t v) {
    if (v == 0) return 0;
    uint64_t p = 1;
    while (p <= v / 2) p <<= 1;
    return p;
}
inline uint64_t ceil_pow2(uint64_t v) {
    uint64_t p = 1;
    while (p < v) p <<= 1;
    return p;
}
inline int log2_exact(uint64_t p) {
    int b = 0;
    while ((1ull << b) < p) b++;
    return b;
}

}  // namespace amj
