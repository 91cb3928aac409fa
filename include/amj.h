/*
 * amj.h - C ABI of the B200-native multi-way join operators (AMHJ multi-way
 * hash join, ALFTJ leapfrog triejoin).
 *
 * Conventions
 *  - Every entry point returns an int status: AMJ_OK (0) or a negative
 *    AMJ_E* code.  amj_last_error() gives a message for the calling thread.
 *    The reference instead logs and calls exit(1) (common-utils/cuda/cuda_base.cuh:43-57).
 *  - No torch types and no CUDA types appear here: streams are `void*`
 *    (a cudaStream_t), device buffers are plain pointers.
 *  - A context (amj_ctx) binds one CUDA device and one stream.  Use one
 *    context per host thread.
 *  - Relations and results are owned by the library until released.
 *  - Attribute values are int32, counts are uint64.  The checksum is defined
 *    in amj_checksum.h.
 *
 * Reference seams replaced (file:line within RapidsAtHKUST/AccMultiwayJoins):
 *  - exec-AMHJ CLI            MHJ-GPU/exec_AMHJ.cu:218-246     -> amj_amhj_execute
 *  - OOC<...>::execute        MHJ-GPU/ooc.cuh:77-82            -> amj_amhj_execute
 *  - exec-LFTJ CLI            LFTJ-GPU/exec_LFTJ.cu:261-268    -> amj_lftj_execute
 *  - OOCWrapper::execute_with_{BFS,DFS}
 *                             LFTJ-GPU/ooc_wrapper.cuh:404-427 -> amj_lftj_execute
 *  - RadixPartitioner::splitKI MHJ-GPU/Indexing/radix_partitioning.cuh:576
 *                                                              -> amj_bucket_build
 *  - constructSortedTrie      LFTJ-GPU/multi_partitioning.cuh:129 -> amj_trie_build
 *  - read_rel_cols_mmap / write_rel_cols_mmap
 *                             common-utils/file_io.h:44-121    -> amj_db_read / amj_db_write
 */
#ifndef AMJ_H
#define AMJ_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- limits (reference: MHJ-GPU/conf.h:22-24, LFTJ-GPU/config.h:16-17) ---- */
#define AMJ_MAX_ATTRS        8   /* attributes in a result tuple             */
#define AMJ_MAX_BUILD_TABLES 6   /* build (hash) tables of one AMHJ query    */
#define AMJ_MAX_COLS         8   /* columns of one relation                  */

/* ---- status codes ---- */
#define AMJ_OK            0
#define AMJ_EINVAL       -1   /* bad argument                                */
#define AMJ_ENOMEM       -2   /* device or host allocation failed            */
#define AMJ_EOVERFLOW    -3   /* a bounded device structure overflowed       */
#define AMJ_ETIMEOUT     -4   /* a bounded device wait ran out               */
#define AMJ_ECUDA        -5   /* a CUDA runtime call failed                  */
#define AMJ_EUNSUPPORTED -6   /* query shape not supported by this operator  */
#define AMJ_EIO          -7   /* file I/O error                              */
#define AMJ_EREJECT      -8   /* admission control rejected the request      */

/* ---- exec-AMHJ query types (MHJ-GPU/exec_AMHJ.cu:5-7) ---- */
#define AMJ_QUERY_NORMAL 0    /* relations given in query order              */
#define AMJ_QUERY_TRI    1    /* triangle over one edge relation             */
#define AMJ_QUERY_FOUR   2    /* 4-clique over one edge relation             */

/* ---- exec-LFTJ algorithm types (LFTJ-GPU/exec_LFTJ.cu:36-39) ---- */
#define AMJ_LFTJ_BFS 0
#define AMJ_LFTJ_DFS 1

/* ---- hash-table layouts for AMHJ build tables ---- */
#define AMJ_LAYOUT_BUCKET    0  /* radix-partitioned bucket CSR (reference default) */
#define AMJ_LAYOUT_OPEN_ADDR 1  /* linear probing, 32-byte-sector slots            */
#define AMJ_LAYOUT_CUCKOO    2  /* bucketised cuckoo, unique keys only             */

/* ---- execute flags ---- */
#define AMJ_F_MATERIALIZE  0x1  /* write the result tuples (else count+checksum) */
#define AMJ_F_HOST_RESULT  0x2  /* copy materialised columns to host memory      */
#define AMJ_F_NO_REORDER   0x4  /* keep fully-bound tables at their query position */
#define AMJ_F_CLIQUE4      0x8  /* amj_lftj_execute, one relation: the 4-clique (the
                                   FOUR pattern) instead of the triangle, DFS only */
#define AMJ_F_KEEP_ORDER   0x10 /* amj_lftj_execute, one relation, and amj_amhj_execute
                                   TRI / FOUR: join the relation as given, never its
                                   degree-ordered copy                              */
#define AMJ_F_DEGREE_ORDER 0x20 /* amj_lftj_execute, one oriented relation: join its
                                   degree-ordered copy (the default for BFS, for DFS
                                   with ws=1 and for the 4-clique; the triangle paths
                                   join it with vertices renamed to their ranks) */
#define AMJ_F_THREAD_PER_ROW 0x80 /* amj_amhj_execute, count only, bucket layout: the
                                   reference's MHJ baseline, one thread per probe row
                                   walking the levels alone (MHJ-GPU/Joins/MHJ.cuh:18) */
#define AMJ_F_PAIRWISE     0x100 /* amj_amhj_execute, NORMAL: a plan of 2-relation joins,
                                   every intermediate result materialised on the device
                                   (the reference's pairwise baseline, MHJ-GPU/exec_PW.cu) */
#define AMJ_F_CLIQUE4_LISTS 0x40 /* amj_lftj_execute with AMJ_F_CLIQUE4: join the
                                   degree-ordered copy by list intersections even where
                                   the triangle matrices fit (same result)          */
#define AMJ_F_FRONTIER     0x400 /* amj_amhj_execute: join every plan with the frontier-DFS
                                   kernel, never the flat kernels of star and canonical
                                   chain count plans (same result; a comparator)   */
#define AMJ_F_HASH_PLAN    0x200 /* amj_amhj_execute, TRI / FOUR over one edge relation:
                                   keep the level-by-level hash-join plan where a bitmap
                                   of b's children (TRI) or the triangle matrices (FOUR)
                                   of the degree-ranked copy would answer the pair-key
                                   levels (same result; those apply to oriented
                                   relations without repeated rows)                 */

/* ---- relation residency ---- */
#define AMJ_MEM_DEVICE 0   /* columns are device pointers, borrowed            */
#define AMJ_MEM_HOST   1   /* columns are host pointers, copied to the device  */
#define AMJ_MEM_HOST_STREAMED 2 /* host columns kept on host (pinned) for ooc  */

typedef struct amj_ctx  amj_ctx;
typedef struct amj_rel  amj_rel;
typedef struct amj_trie amj_trie;
typedef struct amj_batch amj_batch;

typedef struct amj_opts {
    int      block_size;       /* threads per block of the probe kernels (0: 256) */
    int      layout;           /* AMJ_LAYOUT_* for AMHJ build tables              */
    float    load_factor;      /* open addressing load factor (0: 0.5)            */
    int      task_chunk;       /* work-sharing task size in candidates (0: 1024)  */
    uint32_t spin_limit_ms;    /* bound on every device-side wait (0: 5000)       */
    uint64_t task_capacity;    /* work-sharing queue capacity in tasks (0: 1<<22) */
    uint64_t ooc_slice_rows;   /* ooc probe slice rows (0: derived from budget)   */
    uint64_t mem_budget;       /* device bytes the ooc planner may use (0: free/2) */
    uint32_t lftj_heavy_degree; /* ALFTJ ws=1: children count from which a vertex is
                                   joined by the block-wide bitmap kernel (0: 32)  */
    float    dro_headroom;     /* DRO output estimate multiplier (0: 1.05)        */
    uint32_t max_blocks;       /* cap on the blocks of the persistent probe kernels
                                  (0: every block that fits on the device); kernels
                                  of several contexts running at once must fit
                                  together, since idle warps wait for the others  */
    uint32_t lftj_rank_bits;   /* ALFTJ DFS ws=1 over the degree-ranked copy: ranks
                                  each warp's bitmap covers, the highest ones
                                  (0: 32768, the most; rounded up to 32); lower
                                  ranks are found by binary search               */
} amj_opts;

typedef struct amj_result {
    uint64_t count;                   /* bag cardinality                       */
    uint64_t checksum;                /* sum of tuple hashes mod 2^64          */
    int32_t  num_attrs;               /* k, attributes per tuple               */
    int32_t  on_host;                 /* cols[] are host pointers              */
    int32_t *cols[AMJ_MAX_ATTRS];     /* column-major tuples, attribute order  */
    uint64_t rows;                    /* rows present in cols[]                */
    double   build_ms;                /* index build, device time              */
    double   probe_ms;                /* join, device time                     */
    double   total_ms;                /* whole call, device time               */
    uint64_t stats[12];               /* operator counters, see amj_stat_name  */
    double   kernel_ms[4];            /* device time of the main kernels: ALFTJ DFS
                                         [0] rank or bitmap [1] warp intersection, BFS
                                         [0] candidate count [1] expand ([2], [3]
                                         the same in a write pass); AMHJ [0] count
                                         passes [1] write passes; AMHJ with build
                                         relations in host memory (host clock) [0]
                                         partitioning [1] part copies and joins   */
    void    *priv;                    /* library-owned                          */
} amj_result;

/* ---- library / context ---- */
const char *amj_last_error(void);
const char *amj_version(void);
int  amj_ctx_create(int device, const amj_opts *opts, amj_ctx **out);
void amj_ctx_destroy(amj_ctx *ctx);
int  amj_ctx_set_stream(amj_ctx *ctx, void *cuda_stream);
int  amj_ctx_sync(amj_ctx *ctx);
const char *amj_stat_name(int i);
/* number of kernels this context has launched (all entry points) */
int  amj_ctx_launch_count(const amj_ctx *ctx, uint64_t *out);
/* give back what the context keeps between calls for reuse: the pinned host
 * blocks of out-of-core stages and the 4-clique matrix area (both are
 * allocated again when needed) */
int  amj_ctx_trim(amj_ctx *ctx);

/* ---- relations (MHJ-GPU/Relation.cuh:9-38) ---- */
int  amj_rel_create(amj_ctx *ctx, uint64_t n, int ncols, const uint32_t *attrs,
                    const int32_t *const *cols, int where, amj_rel **out);
void amj_rel_release(amj_rel *rel);
int  amj_rel_info(const amj_rel *rel, uint64_t *n, int *ncols, uint32_t *attrs);

/* ---- AMHJ: exec-AMHJ <NORMAL|TRI|FOUR> <path> <ooc> <ws> <dro> <fib> ----
 * NORMAL: rels[0] is the probe relation, rels[1..] the build relations in
 * query order; each build relation is hashed on its first column.  TRI and
 * FOUR take one 2-column edge relation (nrels == 1).  Results follow the
 * multi-attribute compare semantics (every attribute already bound is
 * compared, MHJ-GPU/common_kernels.cuh:41-53).
 * ooc = 1 (OOC::execute, MHJ-GPU/ooc.cuh:77-307): the probe relation is
 * joined in slices; when it is kept in host memory (AMJ_MEM_HOST_STREAMED)
 * the slices are staged on a side stream.  When build relations are kept in
 * host memory too (NORMAL queries), the join runs in stages, one per build
 * relation: the intermediate result and the build relation are
 * hash-partitioned on the key into parts within opts.mem_budget (0: half the
 * free device memory) and joined part by part (stats "slices" counts the
 * part joins).  Relations kept in host memory need ooc = 1. */
int  amj_amhj_execute(amj_ctx *ctx, int query_type, amj_rel *const *rels, int nrels,
                      int ooc, int ws, int dro, int fib, int flags, amj_result *out);

/* ---- ALFTJ: exec-LFTJ <path> <0=BFS|1=DFS> <ooc> <ws> ----
 * nrels == 1: triangle self-join R(a,b) S(b,c) T(a,c) over one edge relation
 *             (AMJ_F_CLIQUE4: the 4-clique).
 * nrels == 3 carrying (0,1), (1,2), (0,2): the triangle over three relations.
 * any other nrels >= 3 (up to 16): the connected join of relations of 1 to 8
 *             columns over attributes 0..k-1, k <= 8 (the reference's LFTJ
 *             stops at 3 attributes and 3 tables of 2 columns).
 * ooc = 1 (every shape; OOCWrapper, LFTJ-GPU/ooc_wrapper.cuh:14-427): the
 *             tries live in pinned host memory (a relation kept on the host,
 *             AMJ_MEM_HOST_STREAMED, has its trie built in value ranges of
 *             its first column); opts.mem_budget (0: half the free device
 *             memory) is split over the attributes that head tries, each
 *             such attribute's values are cut into ranges whose trie slices
 *             fit its share, and every combination of ranges is joined on
 *             the device (stats "slices" counts them).  Relations kept on the
 *             host need ooc = 1.
 * nrels == 2 is rejected, as in the reference (LFTJ-GPU/exec_LFTJ.cu:92-95).
 * 2-column relations are joined as sets (leapfrog triejoin semantics): a
 * repeated row counts once; tries of 3 or more columns keep repeated rows in
 * their last level, as the reference's IndexedTrie does.  The 4-clique over
 * an oriented relation keeps its triangle matrices (at most half the free
 * device memory) with the context between calls; amj_ctx_destroy releases
 * them. */
int  amj_lftj_execute(amj_ctx *ctx, amj_rel *const *rels, int nrels,
                      int algo, int ooc, int ws, int flags, amj_result *out);
/* The same with the attributes bound in attr_order (k entries, a permutation
 * of 0..k-1; null or the identity: amj_lftj_execute), replacing the
 * attr_order argument of OOCWrapper::execute_with_{BFS,DFS}
 * (LFTJ-GPU/ooc_wrapper.cuh:404-427, LFTJ-GPU/ALFTJ.cuh:1125-1196), which the
 * reference's driver always sets to the identity (LFTJ-GPU/exec_LFTJ.cu:230-231).
 * Any order gives the same result: tuples and checksum stay in attribute-id
 * order.  A non-identity order runs the generic join (one relation: its
 * triangle or, with AMJ_F_CLIQUE4, 4-clique pattern); ooc must be 0. */
int  amj_lftj_execute_ordered(amj_ctx *ctx, amj_rel *const *rels, int nrels, int algo, int ooc, int ws,
                              int flags, const uint32_t *attr_order, int k, amj_result *out);

void amj_result_release(amj_result *res);

/* ---- batched AMHJ: many queries, one build pass, one persistent probe launch ----
 * No reference counterpart: the reference runs one query per exec-AMHJ
 * process (MHJ-GPU/exec_AMHJ.cu:218-246).  Queries are compiled as
 * amj_amhj_execute compiles them (same query types, AMJ_F_NO_REORDER
 * allowed) and produce the same count and checksum; they are count-only
 * (no materialisation, ooc, dro or fib).  Relations must stay alive and on
 * the device until the batch is destroyed; their contents may change between
 * runs (a replayed graph reads them again). */
typedef struct amj_batch_opts {
    int      layout;        /* AMJ_LAYOUT_BUCKET or AMJ_LAYOUT_OPEN_ADDR (0: bucket)     */
    float    load_factor;   /* rows per table slot: bucket directory floorPow2(n / lf),
                               open addressing capacity ceilPow2(n / lf)
                               (0: the reference's floorPow2(n) and n / 0.5)             */
    int      block_size;    /* probe threads per block: 128, 256 or 512 (0: 256)        */
    int      task_chunk;    /* work-sharing task size in candidates, >= 32 (0: 1024)   */
    int      use_graph;     /* 1: capture the device sequence into a CUDA graph on the
                               first run with these options and replay it afterwards   */
    int      grid_blocks;   /* probe blocks (0: as many as are resident on the device);
                               a share of the device lets batches run side by side     */
} amj_batch_opts;

typedef struct amj_batch_stats {
    double   build_ms, probe_ms, total_ms;   /* device time of the run               */
    uint64_t launches;                       /* kernels in one run                   */
    uint64_t tasks_pushed, tasks_popped;     /* work-sharing tasks                   */
    uint64_t units;                          /* level-0 units of 1024 candidates     */
    uint64_t build_rows, build_jobs;         /* rows indexed, distinct indexes       */
    int32_t  graph;                          /* 1: the run replayed a captured graph */
    int32_t  pad;
} amj_batch_stats;

/* autotuner grid; a zero count takes the default list
 * (load factor {0.5, 0.7, 0.85}, block {128, 256, 512}, chunk {32 .. 1024}) */
typedef struct amj_batch_tune_grid {
    int   layout;
    int   n_load_factor, n_block_size, n_task_chunk;
    float load_factor[8];
    int   block_size[8];
    int   task_chunk[8];
} amj_batch_tune_grid;

int  amj_batch_create(amj_ctx *ctx, amj_batch **out);
int  amj_batch_submit(amj_batch *b, int query_type, amj_rel *const *rels, int nrels,
                      int flags, uint32_t *qid);
int  amj_batch_size(const amj_batch *b, uint32_t *queries);
/* counts / checksums: one entry per submitted query (either may be NULL) */
int  amj_batch_run(amj_batch *b, const amj_batch_opts *opts, uint64_t *counts,
                   uint64_t *checksums, amj_batch_stats *stats);
/* every grid point on every `sample_every`-th query: one warm-up and `reps`
 * timed runs each; *best gets the point with the least median device time
 * (best->use_graph is kept as passed in) */
int  amj_batch_tune(amj_batch *b, const amj_batch_tune_grid *grid, uint32_t sample_every,
                    int reps, amj_batch_opts *best, double *best_ms);
int  amj_batch_destroy(amj_batch *b);

/* ---- request server: resident relations, continuous batching, ooc spill ----
 * No reference counterpart.  A host thread takes submitted AMHJ queries in
 * arrival order and runs them as batches on `lanes` contexts of the same
 * device (each batch on a share of the SMs, so batches overlap); a request is
 * admitted when its estimated device memory fits the budget left by the
 * batches in flight.  Requests over host-resident relations
 * (AMJ_MEM_HOST_STREAMED), requests submitted with ooc = 1, and requests too
 * large for the whole budget run through the out-of-core operator on their
 * own lane (context, stream and host thread), streaming probe slices from
 * pinned host memory.  The hash indexes of resident relations are kept
 * across requests (the relations must not change while the server runs).
 * Results are the same as one amj_amhj_execute call per query (count and
 * checksum). */
typedef struct amj_server amj_server;

typedef struct amj_serve_opts {
    int      lanes;           /* batches in flight at once (0: 2)                        */
    uint32_t max_batch;       /* queries per batch (0: 256)                               */
    uint64_t mem_budget;      /* device bytes for batches in flight (0: 80% of the free
                                 memory at creation, minus the ooc lane's share)          */
    amj_batch_opts batch;     /* options of every batch (use_graph ignored; grid_blocks 0:
                                 twice the SM count divided by the lanes)                 */
    int      ooc_lane;        /* 1: run out-of-core and spilled requests on their own lane */
    uint64_t ooc_mem;         /* device bytes of the ooc lane's slices (0: free / 8)       */
    uint64_t ooc_slice_rows;  /* ooc probe slice rows (0: derived from ooc_mem)            */
    uint64_t index_cache_bytes; /* device bytes of hash indexes kept across requests (0: 35%
                                   of the free memory at creation)                          */
    int      no_index_cache;  /* 1: build every request's indexes anew                      */
    int      pad;
} amj_serve_opts;

typedef struct amj_serve_result {
    uint64_t count, checksum;
    int32_t  status;          /* AMJ_OK or the error of the request's batch / ooc run */
    int32_t  path;            /* 0 batched, 1 out-of-core lane                         */
    int32_t  spilled;         /* 1: sent to the out-of-core lane by admission           */
    uint32_t batch_id, batch_size;
    int32_t  pad;
    double   queue_ms;        /* submit -> launch                                      */
    double   exec_ms;         /* launch -> result                                      */
    double   latency_ms;      /* submit -> result                                      */
} amj_serve_result;

typedef struct amj_serve_stats {
    uint64_t submitted, completed, rejected, spilled, batches, ooc_runs;
    uint64_t budget_bytes, peak_reserved_bytes;
    uint64_t launches;        /* kernels launched by the lanes and the ooc lane   */
    uint64_t index_hits, index_builds, index_bytes;   /* kept-index cache          */
    uint32_t max_inflight_batches, lanes;
} amj_serve_stats;

int  amj_server_create(amj_ctx *ctx, const amj_serve_opts *opts, amj_server **out);
/* relations must stay alive until the request's result has been waited for */
int  amj_server_submit(amj_server *s, int query_type, amj_rel *const *rels, int nrels,
                       int flags, int ooc, uint64_t *ticket);
/* waits up to timeout_ms (AMJ_ETIMEOUT otherwise); returns the request's
 * status and releases the ticket */
int  amj_server_wait(amj_server *s, uint64_t ticket, uint32_t timeout_ms, amj_serve_result *out);
int  amj_server_stats(amj_server *s, amj_serve_stats *out);
/* finishes every submitted request, then stops the server threads */
int  amj_server_destroy(amj_server *s);

/* ---- building blocks on device pointers, enqueued on the context stream ----
 * amj_bucket_build: bucket-CSR index of n keys with `buckets` (a power of two)
 * buckets, bucket = key & (buckets-1).  Writes hash_keys[n], idx_in_origin[n]
 * (row ids) and buc_ptrs[buckets+1].  Rows inside a bucket are in ascending
 * row order.  (MHJ-GPU/Indexing/radix_partitioning.cuh:576) */
int  amj_bucket_build(amj_ctx *ctx, const int32_t *d_keys, uint64_t n, uint64_t buckets,
                      int32_t *d_hash_keys, uint32_t *d_idx_in_origin, uint32_t *d_buc_ptrs);

/* amj_bucket_build_static: the same bucket-CSR build, for callers that may
 * not allocate device memory (a plugin under an engine that owns all device
 * memory through its own pool, or a latency-critical loop that cannot wait on
 * the driver's allocator).  No counterpart in the reference.  It allocates nothing: its
 * scratch is a fixed area inside the library (about 16.3 MB, resident on
 * every device that loads the library until exit), so n is limited to
 * AMJ_BUCKET_STATIC_MAX_KEYS and buckets to AMJ_BUCKET_STATIC_MAX_BUCKETS
 * (larger requests return AMJ_EINVAL).  Runs on `stream` (a cudaStream_t, 0
 * for the default stream) of the current device and synchronises it before
 * returning.  All calls share the one scratch area: calls that overlap on the
 * GPU race.  The first call on a device looks up the area's address; make it
 * before any stream capture begins. */
#define AMJ_BUCKET_STATIC_MAX_KEYS    (1u << 20)
#define AMJ_BUCKET_STATIC_MAX_BUCKETS (1u << 20)
int  amj_bucket_build_static(const int32_t *d_keys, uint64_t n, uint64_t buckets, int32_t *d_hash_keys,
                             uint32_t *d_idx_in_origin, uint32_t *d_buc_ptrs, void *stream);

/* amj_trie_build: 2-level IndexedTrie of the pairs (c0[i], c1[i]): the
 * distinct c0 values ascending (level 0), their child offsets, and the c1
 * values sorted inside each c0 group (level 1, duplicates kept).
 * (LFTJ-GPU/multi_partitioning.cuh:129-293, LFTJ-GPU/IndexedTrie.cuh:21-31) */
int  amj_trie_build(amj_ctx *ctx, const int32_t *d_c0, const int32_t *d_c1, uint64_t n,
                    amj_trie **out);
/* device views of a trie: level-0 values, level-0 offsets (len0+1 entries),
 * level-1 values */
int  amj_trie_view(const amj_trie *t, uint64_t *len0, uint64_t *len1,
                   const int32_t **d_data0, const uint64_t **d_offsets0,
                   const int32_t **d_data1);
/* copy a trie's three arrays to host memory (len0, len0+1, len1 entries) */
int  amj_trie_download(const amj_trie *t, int32_t *data0, uint64_t *offsets0, int32_t *data1);
/* .tr serialisation, byte layout of IndexedTrie::serialization
 * (LFTJ-GPU/IndexedTrie.cuh:122-156) with attrs {a0,a1} */
int  amj_trie_save(const amj_trie *t, const char *path, uint32_t a0, uint32_t a1);
int  amj_trie_load(amj_ctx *ctx, const char *path, amj_trie **out, uint32_t *a0, uint32_t *a1);
void amj_trie_release(amj_trie *t);

/* N-level tries (1..8 columns), the general IndexedTrie of the reference
 * (LFTJ-GPU/IndexedTrie.cuh:21-209, built by constructSortedTrie for any
 * number of attributes, multi_partitioning.cuh:129-293): level l holds the
 * last values of the distinct (l+1)-prefixes of the lexicographically sorted
 * rows and, except for the last level, the u64 offsets of their children in
 * level l+1 (len[l] + 1 entries); the last level is the sorted last column,
 * duplicates kept.  amj_trie_info / download_level / save_n also accept the
 * 2-level tries of amj_trie_build and amj_trie_load; the .tr layout is the
 * one of amj_trie_save with num_attrs levels. */
int  amj_trie_build_n(amj_ctx *ctx, const int32_t *const *d_cols, int ncols, uint64_t n,
                      amj_trie **out);
int  amj_trie_info(const amj_trie *t, int *levels, uint64_t *lens /* [8] */);
int  amj_trie_download_level(const amj_trie *t, int level, int32_t *data, uint64_t *offsets);
int  amj_trie_save_n(const amj_trie *t, const char *path, const uint32_t *attrs /* [levels] */);
int  amj_trie_load_n(amj_ctx *ctx, const char *path, amj_trie **out, uint32_t *attrs /* [8] */,
                     int *levels);

/* ---- failure detection self-test ----
 * Launches a kernel that waits on a device flag nothing sets.  The wait is
 * bounded by limit_ms (%globaltimer); the call must return AMJ_ETIMEOUT and
 * the context must stay usable.  The same bounded-wait-and-report pattern
 * guards every device-side wait of the operators (work-sharing queue). */
int  amj_selftest_bounded_wait(amj_ctx *ctx, uint32_t limit_ms);

/* ---- seeded synthetic data (host, deterministic, OpenMP) ---- */
int  amj_gen_uniform_i32(int32_t *out, uint64_t n, int64_t lo, int64_t hi_excl,
                         uint64_t seed, uint64_t stream);
int  amj_gen_permutation_i32(int32_t *out, uint64_t n, uint64_t seed, uint64_t stream);
/* Zipf(theta) ranks over [0, domain); rank r maps to rank_to_key[r] when given */
int  amj_gen_zipf_i32(int32_t *out, uint64_t n, uint64_t domain, double theta,
                      const int32_t *rank_to_key, uint64_t seed, uint64_t stream);
/* R-MAT graph: nedges draws with quadrant probabilities (a,b,c,1-a-b-c) over
 * 2^scale vertices; self-loops dropped, edges oriented u<v, duplicates
 * removed, then shuffled.  src/dst need room for nedges; *n_out = E'. */
int  amj_gen_rmat(int scale, uint64_t nedges, double a, double b, double c, uint64_t seed,
                  int32_t *src, int32_t *dst, uint64_t *n_out);

/* ---- .db files: column-major int32, name "<rows>_<attr0>_<attr1>...db" ---- */
int  amj_db_write(const char *path, uint64_t n, int ncols, const int32_t *const *cols);
int  amj_db_read(const char *path, uint64_t n, int ncols, int32_t *const *cols);
int  amj_db_parse_name(const char *path, uint64_t *n, int *ncols, uint32_t *attrs);

/* ---- edge-list text converters ----
 * An edge list is a text file of one edge per line: two integers separated by
 * any run of ' ', '|' or tab; each value is stored as int32 modulo 2^32 (the
 * reference's stoul-then-int).  Blank lines and lines starting with '#' or '%'
 * are skipped; any other line must hold exactly two integers (AMJ_EINVAL
 * names the first that does not).  swap != 0 reverses the two columns
 * (MHJ-GPU/switch_el.py).
 * amj_edgelist_read: the edges into src/dst (cap rows available; cap = 0 only
 *   sets *n, the number of edges).
 * amj_edgelist_to_db: the edges as a 2-column .db file (column-major int32),
 *   replacing edgelist_2_db (MHJ-GPU/exec_el_2_db.cu:20-87), which writes
 *   "<edgelist>.db".
 * amj_edgelist_to_tr: the 2-level trie of the edges (amj_trie_build, level 1
 *   keeps repeated rows) saved as a .tr file with attributes (0, 1), replacing
 *   edgelist_to_csr (LFTJ-GPU/edgelist_to_csr.cu:19-86), which writes
 *   "output.tr". */
int  amj_edgelist_read(const char *path, int swap, int32_t *src, int32_t *dst, uint64_t cap, uint64_t *n);
int  amj_edgelist_to_db(const char *text_path, const char *db_path, int swap, uint64_t *rows);
int  amj_edgelist_to_tr(amj_ctx *ctx, const char *text_path, const char *tr_path, int swap, uint64_t *rows);
/* amj_tbl_to_db: fields fields[0..ncols-1] (0-based, any order) of a
 * delimited table (runs of tab, '|' or newline separate fields; a selected
 * field is read as stoul does: its leading integer) as a .db file named
 * "<rows>_<attrs[0]>_<attrs[1]>...db" in out_dir (null: the current
 * directory); its path goes to out_path (out_cap bytes).  Blank lines are
 * skipped; a line missing a selected field, or one that is not an integer,
 * is an error naming the line.  Replaces tbl_2_db
 * (MHJ-GPU/exec_tbl_2_db.cu:26-133), the ingestion of TPC-H .tbl files. */
int  amj_tbl_to_db(const char *tbl_path, const uint32_t *fields, const uint32_t *attrs, int ncols,
                   const char *out_dir, char *out_path, uint64_t out_cap, uint64_t *rows);

/* ---- host checksum of column-major tuples (same definition as the GPU) ---- */
int  amj_checksum_host(const int32_t *const *cols, int k, uint64_t n, uint64_t *out);

#ifdef __cplusplus
}
#endif
#endif /* AMJ_H */
