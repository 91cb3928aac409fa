// Test infrastructure only: drives the reference's MHJ-CPU (pthreads
// multi-way hash join, MHJ-CPU/MHJ.cpp) from its own source files, compiled
// where they lie, so tests and the CPU baseline can run the reference itself.
// Nothing in the product library links or loads this file's output.
//
// MHJ.cpp calls a misnamed MHJ<> from test_general (MHJ.cpp:579) although the
// function is TBJ (MHJ.cpp:378): MHJ is defined to TBJ.  Its main() is
// renamed.  TBJ returns only the count and keeps its result chunks in an
// array it passes to every worker thread (MHJ.cpp:404-407, 469); the harness
// sees that array by wrapping pthread_create, then walks the chunks to get
// the tuples and their checksum, and frees them.
#include <pthread.h>
#include <chrono>
#include <cstring>   // MHJ.cpp relies on log.h for <cstring>, which logging off leaves out
#include <cstdint>
#include <vector>

extern "C" int amj_ref_hook_pthread_create(pthread_t *, const pthread_attr_t *, void *(*)(void *), void *);

#define pthread_create amj_ref_hook_pthread_create
#define main mhj_ref_main
#define MHJ TBJ
#include "MHJ.cpp"
#undef pthread_create
#undef main

#include "../../include/amj_checksum.h"

using RefRel = Relation<int, unsigned long long>;
using RefChunk = ResChunk<int, unsigned long long>;
using RefArgs = TBJ_arg_t<int, unsigned long long>;

static RefChunk **g_join_res = nullptr;
static int g_nthreads = 0;

extern "C" int amj_ref_hook_pthread_create(pthread_t *t, const pthread_attr_t *a, void *(*f)(void *), void *arg) {
    const RefArgs *args = (const RefArgs *)arg;
    g_join_res = args->m_join_res;
    g_nthreads = args->m_nthreads;
    return pthread_create(t, a, f, arg);
}

// Run TBJ on `ntables` relations in query order (table 0 probes).
// attrs: ntables x 8 attribute ids, data: ntables x 8 column pointers.
// Returns 0, or -1 when the attributes are not 0..k-1.  When tuples is not
// null, up to cap tuples are copied column-major (k columns, attribute order).
extern "C" int mhjref_run(int ntables, const uint64_t *lens, const int *ncols, const uint32_t *attrs,
                          const int32_t *const *data, int nthreads, uint64_t *count, uint64_t *checksum,
                          int32_t *const *tuples, uint64_t cap, int *k_out, double *seconds) {
    std::vector<RefRel> rels(ntables);
    bool seen[MAX_NUM_RES_ATTRS] = {false};
    int k = 0, n_iRes = 0;
    std::vector<AttrType> iRes_attrs(MAX_NUM_RES_ATTRS);
    std::vector<bool *> used(ntables - 1);
    for (int i = 0; i < ntables; i++) {
        rels[i].init((uint32_t)ncols[i], lens[i]);
        if (i) used[i - 1] = (bool *)malloc(sizeof(bool) * ncols[i]);
        for (int c = 0; c < ncols[i]; c++) {
            const uint32_t a = attrs[i * 8 + c];
            if (a >= MAX_NUM_RES_ATTRS) return -1;
            rels[i].attr_list[c] = a;
            rels[i].data[c] = const_cast<int32_t *>(data[i * 8 + c]);
            if (!seen[a]) {
                seen[a] = true;
                k++;
                if (i) used[i - 1][c] = false;
                if (i != ntables - 1) iRes_attrs[n_iRes++] = a;
            } else if (i) {
                used[i - 1][c] = true;
            }
        }
    }
    for (int a = 0; a < k; a++)
        if (!seen[a]) return -1;
    std::vector<unsigned long long> buckets;
    for (int i = 1; i < ntables; i++) buckets.push_back(floorPowerOf2<unsigned long long>(rels[i].length / BUC_RATIO));
    g_join_res = nullptr;
    auto t0 = std::chrono::steady_clock::now();
    unsigned long long n = TBJ<int, unsigned long long>(rels, used, buckets, iRes_attrs, n_iRes, k, nthreads);
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    uint64_t sum = 0, pos = 0;
    for (int t = 0; g_join_res && t < g_nthreads; t++) {
        RefChunk *ch = g_join_res[t];
        while (ch) {
            for (unsigned long long r = 0; r < ch->num_res; r++) {
                uint64_t h = AMJ_CHECKSUM_SEED;
                for (int a = 0; a < k; a++) h = amj_hash_step(h, ch->data[a][r]);
                sum += h;
                if (tuples && pos < cap)
                    for (int a = 0; a < k; a++) tuples[a][pos] = ch->data[a][r];
                pos++;
            }
            RefChunk *next = ch->next;
            for (uint32_t a = 0; a < ch->num_res_attrs; a++) free(ch->data[a]);
            free(ch->data);
            delete ch;
            ch = next;
        }
    }
    if (g_join_res) delete[] g_join_res;
    g_join_res = nullptr;
    for (auto *u : used) free(u);
    for (auto &r : rels) r.destroy();
    *count = n;
    *checksum = sum;
    if (k_out) *k_out = k;
    return pos == n ? 0 : -2;
}
