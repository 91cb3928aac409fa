// Host-side AMHJ plan types shared by the single-query operator (amhj.cu)
// and the batched executor (amhj_batch.cu).
#pragma once
#include "amhj_kernel.cuh"

#include <tuple>

namespace amj {

struct LevelSpec {
    const amj_rel *rel;
    int ncols;
    int src_col[4];    // relation column feeding index column c (index column 0 is the key)
    int attr[4];       // attribute of index column c
    int key_mode;
    uint8_t cmp_mask, bind_mask;
};

struct HostPlan {
    const amj_rel *probe = nullptr;
    int probe_attr[AMJ_MAX_COLS] = {};
    int L = 0, k = 0;
    LevelSpec lv[AMJ_MAX_BUILD_TABLES];
};

struct IndexKey {
    const amj_rel *rel;
    int src[4];
    int ncols, key_mode, layout;
    uint64_t uid = 0;   // the relation's serial number: a reused address is another relation
    float load_factor = 0.f;
    bool operator<(const IndexKey &o) const {
        return std::tie(uid, rel, src[0], src[1], src[2], src[3], ncols, key_mode, layout, load_factor) <
               std::tie(o.uid, o.rel, o.src[0], o.src[1], o.src[2], o.src[3], o.ncols, o.key_mode, o.layout,
                        o.load_factor);
    }
};

// Indexes kept across calls.  get() returns a complete index of the level's
// relation columns (built on ctx's stream and synchronised on a miss), or
// null when the provider keeps no index for it (the caller builds its own).
struct IndexProvider {
    virtual ~IndexProvider() = default;
    virtual const HashIndex *get(amj_ctx *ctx, const IndexKey &key, const LevelSpec &ls) = 0;
};

// Level descriptor of a complete index.
void fill_level_from_index(const LevelSpec &ls, const HashIndex &ix, LevelDesc *d);

// Compile a query (reference exec_AMHJ.cu:70-89, TRI/FOUR :32-69) into the
// probe relation and the ordered build levels.
int compile_plan(int query_type, amj_rel *const *rels, int nrels, int flags, HostPlan *hp);

// Level descriptor of index `layout` over the given device arrays.
void fill_level_desc(const LevelSpec &ls, int layout, int key_mode, uint32_t mask, const uint32_t *buc_ptrs,
                     const int32_t *const *cols, const int2 *slots, LevelDesc *d);

// Plan fields that depend only on the query and the options (levels excluded).
void plan_common(const HostPlan &hp, const amj_opts &o, ProbePlan *P);

// ooc = 1 with build relations in host memory: the join in stages, each a
// hash partition of the intermediate result and one build relation into
// parts that fit the memory budget, joined part by part (amhj_partitioned.cu).
int amhj_partitioned_execute(amj_ctx *ctx, const HostPlan &hp, int ws, int dro, int flags, amj_result *out);
// AMJ_F_PAIRWISE: the plan as 2-relation joins with materialised intermediates.
int amhj_pairwise_execute(amj_ctx *ctx, const HostPlan &hp, int ws, int dro, int flags, amj_result *out);
// FOUR over one oriented edge relation without repeated rows through the
// triangle matrices of its degree-ranked copy (lftj_api.cu); *used is false
// where they do not apply.
int amhj_four_by_matrices(amj_ctx *ctx, amj_rel *rel, int flags, amj_result *out, bool *used);
// TRI over one edge relation through the wedge kernel on its degree-ranked
// copy (lftj_api.cu); *used is false where that does not apply.
int amhj_tri_by_wedges(amj_ctx *ctx, amj_rel *rel, int flags, amj_result *out, bool *used);

}  // namespace amj
