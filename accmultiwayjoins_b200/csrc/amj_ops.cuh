// Index structures and operator entry points shared between the translation
// units of libamj.
#pragma once
#include "amj_cuda.cuh"

struct ResultOwner {
    amj_ctx *ctx = nullptr;
};

namespace amj {

void result_init(amj_result *res, int k);

// Key of a hash index: the build relation's first column, or the pair of
// its first two columns (used when every column of the build relation is
// already bound at its level, i.e. the table only filters).
enum KeyMode : int { KEY_SINGLE = 0, KEY_PAIR = 1 };

constexpr int32_t OA_EMPTY_KEY = INT32_MIN;   // open addressing / cuckoo empty slot marker
constexpr int CUCKOO_SLOTS = 4;                // slots per cuckoo bucket (one 32-byte sector)

// A hash index over a build relation with at most 4 columns.  For the bucket
// layout the relation's columns are stored in bucket order next to each other
// (structure of arrays) so a probe reads the key and the bound payload from
// the same position: no row-id indirection into the original relation, unlike
// the reference's hash_keys / idx_in_origin / data[] triple
// (MHJ-GPU/Relation.cuh:50-63).  Open addressing and cuckoo store (c0, c1)
// pairs in 8-byte slots, four to a 32-byte sector.
struct HashIndex {
    int layout = AMJ_LAYOUT_BUCKET;
    int key_mode = KEY_SINGLE;
    uint64_t n = 0;
    int ncols = 0;
    uint32_t mask = 0;             // buckets-1, capacity-1, or cuckoo buckets-1
    DBuf<uint32_t> buc_ptrs;       // bucket layout: buckets+1 offsets
    DBuf<int32_t> cols[4];         // bucket layout: columns in bucket order
    DBuf<int2> slots;              // open addressing / cuckoo
};

int build_hash_index(amj_ctx *ctx, const int32_t *const *d_cols, int ncols, uint64_t n, int layout,
                     int key_mode, float load_factor, HashIndex *out);

// 2-level trie (CSR): level 0 distinct first-column values, offsets into
// level 1, level 1 second-column values sorted within each group.
struct Trie2 {
    uint64_t len0 = 0, len1 = 0;
    DBuf<int32_t> data0;
    DBuf<uint64_t> off0;
    DBuf<int32_t> data1;
    DBuf<int32_t> src1;        // level-0 value of every level-1 entry (sorted first column)
    DBuf<uint64_t> rowptr;     // dense child offsets for values rp_min .. rp_min+rp_count-1 (+1 end entry)
    int32_t rp_min = 0;
    uint64_t rp_count = 0;     // 0 when no dense array was built
};

// Level 1 of a built 2-level trie has TRIE_LEVEL1_PAD spare values after its
// last one, so kernels may read it in aligned 16-byte quads.
constexpr uint64_t TRIE_LEVEL1_PAD = 4;
// distinct: drop repeated rows (the set semantics of the leapfrog triejoin);
// vmax >= 0: every value of both columns lies in [0, vmax] (no min/max pass)
int build_trie2(amj_ctx *ctx, const int32_t *d_c0, const int32_t *d_c1, uint64_t n, Trie2 *out,
                bool distinct = false, int32_t vmax = -1);
// The distinct 2-level trie of a degree-ranked copy: every value in [0, nv)
// and each row's first value below its second (rows bucketed by counting,
// each row sorted on its own; the radix-sort build where a row is too long).
int build_trie2_ranked(amj_ctx *ctx, const int32_t *d_c0, const int32_t *d_c1, uint64_t n, uint64_t nv, Trie2 *out);

// time between two events recorded on the context stream (ms)
double event_ms(cudaEvent_t a, cudaEvent_t b);

// Degree-ordered copy (ns, nd) of the edge relation (c0, c1) when every edge
// has 0 <= c0 < c1 (*oriented); otherwise nothing is allocated.
int degree_ordered_copy(amj_ctx *ctx, const int32_t *c0, const int32_t *c1, uint64_t n, DBuf<int32_t> *ns,
                        DBuf<int32_t> *nd, bool *oriented);

// The same copy with every vertex renamed to its rank in (degree, id) order:
// edges (rank lo, rank hi), *inv[rank] = the vertex id, *nv ranks.
int degree_ranked_copy(amj_ctx *ctx, const int32_t *c0, const int32_t *c1, uint64_t n, DBuf<int32_t> *ns,
                       DBuf<int32_t> *nd, DBuf<int32_t> *inv, uint64_t *nv, bool *oriented);
// The ranks alone: *rank[id] and *inv[rank] over ids 0..*nv-1 (when oriented).
int degree_ranks(amj_ctx *ctx, const int32_t *c0, const int32_t *c1, uint64_t n, DBuf<int32_t> *rank,
                 DBuf<int32_t> *inv, uint64_t *nv, bool *oriented);
// The level-1 entries of a degree-ranked trie grouped by b (a stable sort).
int build_wedges(amj_ctx *ctx, const Trie2 &R, uint64_t nv, DBuf<uint64_t> *out);

// copy materialised device result columns to pinned host memory (when asked)
int finish_result_columns(amj_ctx *ctx, amj_result *res, int flags);

}  // namespace amj

namespace amj {
constexpr int TRIE_MAX_LEVELS = 8;

// N-level trie: level l holds the last values of the distinct (l+1)-prefixes
// of the sorted rows, off[l] the offsets of their children in level l+1; the
// last level is the sorted last column, duplicates kept.
struct TrieN {
    int levels = 0;
    uint64_t len[TRIE_MAX_LEVELS] = {};
    DBuf<int32_t> data[TRIE_MAX_LEVELS];
    DBuf<uint64_t> off[TRIE_MAX_LEVELS - 1];
};

int build_trieN(amj_ctx *ctx, const int32_t *const *d_cols, int ncols, uint64_t n, TrieN *out);
}  // namespace amj

// A trie handle: a 2-level trie (t, levels = 0 in tn) or an N-level one (tn).
struct amj_trie {
    amj_ctx *ctx = nullptr;
    amj::Trie2 t;
    amj::TrieN tn;
    int levels() const { return tn.levels ? tn.levels : 2; }
    uint64_t len(int l) const { return tn.levels ? tn.len[l] : (l == 0 ? t.len0 : t.len1); }
    const int32_t *data(int l) const { return tn.levels ? tn.data[l].p : (l == 0 ? t.data0.p : t.data1.p); }
    const uint64_t *off(int l) const { return tn.levels ? tn.off[l].p : t.off0.p; }
};
