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

#ifdef AMJ_REF_MULTI_KEY
// Multi-key build (-DAMJ_REF_MULTI_KEY, _ref/libmhjref_mk.so).  The reference's
// probe has a branch that compares every already-bound attribute of a build
// tuple (probe_tbj / probe_write with single_join_key = false, MHJ.cpp:64-90,
// :205-245), which is the semantics of cyclic queries (TRI, FOUR).  prj_thread
// only ever instantiates the single-key branch (MHJ.cpp:367).  Without editing
// the reference, this build declares an explicit specialisation of the
// single-key instantiation before MHJ.cpp is read, and defines it after as a
// call to the multi-key instantiation: every TBJ call then runs the
// reference's own multi-key probe.
template <typename DataType, typename CntType> struct TBJ_arg_t;
template <typename DataType, typename CntType, bool single_join_key>
void probe_write(TBJ_arg_t<DataType, CntType> *args);
template <> void probe_write<int, unsigned long long, true>(TBJ_arg_t<int, unsigned long long> *args);
#define AMJ_REF_ENTRY mhjref_run_mk
#else
#define AMJ_REF_ENTRY mhjref_run
#endif

#define pthread_create amj_ref_hook_pthread_create
#define main mhj_ref_main
#define MHJ TBJ
#include "MHJ.cpp"
#undef pthread_create
#undef main

#ifdef AMJ_REF_MULTI_KEY
template <> void probe_write<int, unsigned long long, true>(TBJ_arg_t<int, unsigned long long> *args) {
    probe_write<int, unsigned long long, false>(args);
}
#endif

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
// relabel (optional, nlabels entries): every result value v is replaced by
// relabel[v] and the values of each tuple are then sorted ascending before
// the tuple is hashed or copied (-3 when a value lies outside the map).  A
// triangle or 4-clique query joined over a vertex-renamed copy of an edge
// relation, oriented from lower to higher new name, lists the same cliques
// as the query over the relation oriented u < v; renamed back and sorted,
// its tuples are those of the original query.
static int run_impl(int ntables, const uint64_t *lens, const int *ncols, const uint32_t *attrs,
                    const int32_t *const *data, int nthreads, uint64_t *count, uint64_t *checksum,
                    int32_t *const *tuples, uint64_t cap, int *k_out, double *seconds, const int32_t *relabel,
                    uint64_t nlabels) {
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
            if (a >= MAX_NUM_RES_ATTRS) {
                for (auto *u : used) free(u);
                return -1;
            }
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
        if (!seen[a]) {
            for (auto *u : used) free(u);
            return -1;
        }
    std::vector<unsigned long long> buckets;
    for (int i = 1; i < ntables; i++) buckets.push_back(floorPowerOf2<unsigned long long>(rels[i].length / BUC_RATIO));
    g_join_res = nullptr;
    auto t0 = std::chrono::steady_clock::now();
    unsigned long long n = TBJ<int, unsigned long long>(rels, used, buckets, iRes_attrs, n_iRes, k, nthreads);
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    uint64_t sum = 0, pos = 0;
    bool bad_label = false;
    for (int t = 0; g_join_res && t < g_nthreads; t++) {
        RefChunk *ch = g_join_res[t];
        while (ch) {
            for (unsigned long long r = 0; r < ch->num_res; r++) {
                int32_t v[MAX_NUM_RES_ATTRS];
                for (int a = 0; a < k; a++) v[a] = ch->data[a][r];
                if (relabel) {
                    for (int a = 0; a < k; a++) {
                        if (v[a] < 0 || (uint64_t)v[a] >= nlabels) {
                            bad_label = true;
                            v[a] = 0;
                        } else {
                            v[a] = relabel[v[a]];
                        }
                    }
                    for (int a = 1; a < k; a++)  // insertion sort of <= 8 values
                        for (int b = a; b > 0 && v[b - 1] > v[b]; b--) std::swap(v[b - 1], v[b]);
                }
                sum += amj_tuple_hash_k(v, k);
                if (tuples && pos < cap)
                    for (int a = 0; a < k; a++) tuples[a][pos] = v[a];
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
    if (bad_label) return -3;
    return pos == n ? 0 : -2;
}

#define AMJ_REF_CAT2(a, b) a##b
#define AMJ_REF_CAT(a, b) AMJ_REF_CAT2(a, b)

extern "C" int AMJ_REF_ENTRY(int ntables, const uint64_t *lens, const int *ncols, const uint32_t *attrs,
                             const int32_t *const *data, int nthreads, uint64_t *count, uint64_t *checksum,
                             int32_t *const *tuples, uint64_t cap, int *k_out, double *seconds) {
    return run_impl(ntables, lens, ncols, attrs, data, nthreads, count, checksum, tuples, cap, k_out, seconds,
                    nullptr, 0);
}

// The same with the result renamed through `relabel` and sorted per tuple.
extern "C" int AMJ_REF_CAT(AMJ_REF_ENTRY, _relabel)(int ntables, const uint64_t *lens, const int *ncols,
                                                    const uint32_t *attrs, const int32_t *const *data,
                                                    int nthreads, uint64_t *count, uint64_t *checksum,
                                                    int32_t *const *tuples, uint64_t cap, int *k_out,
                                                    double *seconds, const int32_t *relabel, uint64_t nlabels) {
    if (!relabel) return -1;
    return run_impl(ntables, lens, ncols, attrs, data, nthreads, count, checksum, tuples, cap, k_out, seconds,
                    relabel, nlabels);
}
