/*
 * amj_oracle.c - CPU restatement of the reference's join semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  The parity tests, __graft_entry__.smoke() and
 * the CPU-baseline leg of bench.py call these functions as the checker; the
 * product library (libamj) never links, loads or calls them.
 *
 * Parity is pinned by the reference itself: orc_mhj must agree with the
 * reference's MHJ-CPU (oracle/_ref/libmhjref.so, built from
 * MHJ-CPU/MHJ.cpp) on chain and star queries, and the triangle / 4-clique
 * restatements must agree with orc_mhj on the TRI / FOUR attribute patterns.
 * The reference ships no golden vectors; the fixtures under tests/golden/
 * are outputs of MHJ-CPU run here.
 *
 * Functions
 *  orc_bucket_build  bucket CSR of keys, bucket = key & (B-1), rows in row
 *                    order (what RadixPartitioner::splitKI produces up to the
 *                    order inside a bucket, MHJ-GPU/Indexing/radix_partitioning.cuh:508-578)
 *  orc_trie_build    2-level IndexedTrie (LFTJ-GPU/multi_partitioning.cuh:129-293)
 *  orc_trie_build_n  the same for 1..8 columns: rows sorted lexicographically;
 *                    level l holds the distinct (l+1)-prefixes' last values and
 *                    the offsets of their children in level l+1; the last level
 *                    is the sorted last column, duplicates kept
 *  orc_mhj           multi-way hash join, depth-first with backtracking per
 *                    probe row (MHJ-CPU/MHJ.cpp:176-279) comparing every bound
 *                    attribute (the multi-key compare of
 *                    MHJ-GPU/common_kernels.cuh:41-53)
 *  orc_triangle      R(a,b) S(b,c) T(a,c) over one edge relation, bag
 *                    semantics, by sorted adjacency merges (the answer of
 *                    ALFTJ on LFTJ-GPU/exec_LFTJ.cu:218-222's attribute lists)
 *  orc_four_clique   the FOUR pattern (MHJ-GPU/exec_AMHJ.cu:59-64) over a
 *                    set of edges oriented u < v
 * All return counts, the checksum of include/amj_checksum.h and optionally
 * the tuples (column-major, attribute order).
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/amj_checksum.h"

#define ORC_MAX_ATTRS 8
#define ORC_MAX_RELS 8

static uint64_t floor_pow2(uint64_t v) {
    uint64_t p = 1;
    if (v == 0) return 1;
    while (p <= v / 2) p <<= 1;
    return p;
}

int orc_bucket_build(const int32_t *keys, uint64_t n, uint64_t B, int32_t *hash_keys, uint32_t *idx,
                     uint32_t *buc_ptrs) {
    if (B == 0 || (B & (B - 1))) return -1;
    memset(buc_ptrs, 0, (B + 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < n; i++) buc_ptrs[((uint32_t)keys[i] & (B - 1)) + 1]++;
    for (uint64_t b = 0; b < B; b++) buc_ptrs[b + 1] += buc_ptrs[b];
    uint32_t *pos = (uint32_t *)malloc((B + 1) * sizeof(uint32_t));
    if (!pos) return -2;
    memcpy(pos, buc_ptrs, (B + 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < n; i++) {
        uint32_t b = (uint32_t)keys[i] & (uint32_t)(B - 1);
        if (hash_keys) hash_keys[pos[b]] = keys[i];
        if (idx) idx[pos[b]] = (uint32_t)i;
        pos[b]++;
    }
    free(pos);
    return 0;
}

static int cmp_i64(const void *a, const void *b) {
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return x < y ? -1 : x > y;
}

/* pack (c0, c1) so that signed int64 order is (c0, c1) lexicographic order:
 * c0 in the high half keeps its two's-complement sign bit, c1 in the low half
 * is sign-flipped so its unsigned magnitude orders like the signed value */
static int64_t pack_pair(int32_t a, int32_t b) {
    return (int64_t)(((uint64_t)(uint32_t)a << 32) | ((uint32_t)b ^ 0x80000000u));
}
static int32_t pair_c0(int64_t p) { return (int32_t)(uint32_t)((uint64_t)p >> 32); }
static int32_t pair_c1(int64_t p) { return (int32_t)((uint32_t)(uint64_t)p ^ 0x80000000u); }

/* lexicographic order of rows over ncols columns (qsort context through a static) */
static const int32_t *const *g_tn_cols;
static int g_tn_ncols;
static int cmp_rows(const void *a, const void *b) {
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    for (int c = 0; c < g_tn_ncols; c++) {
        const int32_t u = g_tn_cols[c][x], v = g_tn_cols[c][y];
        if (u != v) return u < v ? -1 : 1;
    }
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* data[l] must hold n values and off[l] n + 1 (l < ncols - 1); len[l] gets
   the number of values of level l.  Not reentrant (qsort context). */
int orc_trie_build_n(const int32_t *const *cols, int ncols, uint64_t n, int32_t *const *data, uint64_t *const *off,
                     uint64_t *len) {
    if (ncols < 1 || ncols > ORC_MAX_ATTRS) return -1;
    uint64_t *perm = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
    if (!perm) return -2;
    for (uint64_t i = 0; i < n; i++) perm[i] = i;
    g_tn_cols = cols;
    g_tn_ncols = ncols;
    qsort(perm, n, sizeof(uint64_t), cmp_rows);
    /* cnt[l]: nodes of level l so far */
    uint64_t cnt[ORC_MAX_ATTRS] = {0};
    for (uint64_t i = 0; i < n; i++) {
        int changed = i == 0;
        for (int l = 0; l < ncols; l++) {
            if (!changed && cols[l][perm[i]] != cols[l][perm[i - 1]]) changed = 1;
            if (l == ncols - 1) {
                data[l][i] = cols[l][perm[i]];
                continue;
            }
            if (changed) {
                /* a new node at level l; its first child is the next node of level l+1 */
                data[l][cnt[l]] = cols[l][perm[i]];
                off[l][cnt[l]] = (l + 1 == ncols - 1) ? i : cnt[l + 1];
                cnt[l]++;
            }
        }
    }
    for (int l = 0; l + 1 < ncols; l++) {
        off[l][cnt[l]] = (l + 1 == ncols - 1) ? n : cnt[l + 1];
        len[l] = cnt[l];
    }
    len[ncols - 1] = n;
    free(perm);
    return 0;
}

int orc_trie_build(const int32_t *c0, const int32_t *c1, uint64_t n, int32_t *data0, uint64_t *off0, int32_t *data1,
                   uint64_t *len0) {
    int64_t *p = (int64_t *)malloc((n ? n : 1) * sizeof(int64_t));
    if (!p) return -2;
    for (uint64_t i = 0; i < n; i++) p[i] = pack_pair(c0[i], c1[i]);
    qsort(p, n, sizeof(int64_t), cmp_i64);
    uint64_t m = 0;
    for (uint64_t i = 0; i < n; i++) {
        data1[i] = pair_c1(p[i]);
        if (i == 0 || pair_c0(p[i]) != pair_c0(p[i - 1])) {
            data0[m] = pair_c0(p[i]);
            off0[m] = i;
            m++;
        }
    }
    off0[m] = n;
    *len0 = m;
    free(p);
    return 0;
}

/* ------------------------------------------------------------------ mhj -- */

typedef struct {
    uint64_t n;
    int ncols;
    int attr[ORC_MAX_ATTRS];
    const int32_t *col[ORC_MAX_ATTRS];
} orc_rel;

typedef struct {
    const orc_rel *r;
    uint64_t B;
    uint32_t *buc;   /* B+1 offsets */
    uint32_t *rows;  /* rows in bucket order */
    int key_bound;   /* column 0 bound before this level: bucket lookup, else full scan */
    int cmp[ORC_MAX_ATTRS];
} orc_level;

typedef struct {
    int L, k;
    orc_level lv[ORC_MAX_RELS];
    uint64_t cnt, sum;
    int32_t *const *tuples;
    uint64_t cap;
    uint64_t *pos; /* shared output cursor */
} orc_walk;

static void orc_emit(orc_walk *w, const int32_t *iRes) {
    uint64_t h = AMJ_CHECKSUM_SEED;
    for (int a = 0; a < w->k; a++) h = amj_hash_step(h, iRes[a]);
    w->cnt++;
    w->sum += h;
    if (w->tuples) {
        uint64_t p;
#pragma omp atomic capture
        p = (*w->pos)++;
        if (p < w->cap)
            for (int a = 0; a < w->k; a++) w->tuples[a][p] = iRes[a];
    }
}

static void orc_dfs(orc_walk *w, int level, int32_t *iRes) {
    if (level == w->L) {
        orc_emit(w, iRes);
        return;
    }
    const orc_level *lv = &w->lv[level];
    const orc_rel *r = lv->r;
    uint64_t s = 0, e = r->n;
    if (lv->key_bound) {
        uint32_t b = (uint32_t)iRes[r->attr[0]] & (uint32_t)(lv->B - 1);
        s = lv->buc[b];
        e = lv->buc[b + 1];
    }
    for (uint64_t i = s; i < e; i++) {
        uint64_t row = lv->key_bound ? lv->rows[i] : i;
        int ok = 1;
        for (int c = 0; c < r->ncols && ok; c++)
            if (lv->cmp[c] && r->col[c][row] != iRes[r->attr[c]]) ok = 0;
        if (!ok) continue;
        int32_t saved[ORC_MAX_ATTRS];
        memcpy(saved, iRes, sizeof(saved));
        for (int c = 0; c < r->ncols; c++)
            if (!lv->cmp[c]) iRes[r->attr[c]] = r->col[c][row];
        orc_dfs(w, level + 1, iRes);
        memcpy(iRes, saved, sizeof(saved));
    }
}

/* rels[0] probes; rels[1..] are joined in the given order.  Returns 0, -1 on a
 * bad query (attributes not 0..k-1), -2 on allocation failure. */
int orc_mhj(int nrels, const orc_rel *rels, int nthreads, uint64_t *count, uint64_t *checksum,
            int32_t *const *tuples, uint64_t cap) {
    if (nrels < 1 || nrels > ORC_MAX_RELS) return -1;
    orc_walk base;
    memset(&base, 0, sizeof(base));
    uint32_t seen = 0;
    for (int i = 0; i < nrels; i++)
        for (int c = 0; c < rels[i].ncols; c++) {
            if (rels[i].attr[c] < 0 || rels[i].attr[c] >= ORC_MAX_ATTRS) return -1;
            seen |= 1u << rels[i].attr[c];
        }
    int k = 0;
    while (k < 32 && ((seen >> k) & 1)) k++;
    if (seen != ((1u << k) - 1)) return -1;
    base.k = k;
    base.L = nrels - 1;
    uint32_t bound = 0;
    for (int c = 0; c < rels[0].ncols; c++) bound |= 1u << rels[0].attr[c];
    int rc = 0;
    for (int l = 0; l < base.L; l++) {
        orc_level *lv = &base.lv[l];
        const orc_rel *r = &rels[l + 1];
        lv->r = r;
        for (int c = 0; c < r->ncols; c++) lv->cmp[c] = (bound >> r->attr[c]) & 1;
        lv->key_bound = lv->cmp[0];
        lv->B = floor_pow2(r->n);
        lv->buc = (uint32_t *)malloc((lv->B + 1) * sizeof(uint32_t));
        lv->rows = (uint32_t *)malloc((r->n ? r->n : 1) * sizeof(uint32_t));
        if (!lv->buc || !lv->rows) rc = -2;
        else orc_bucket_build(r->col[0], r->n, lv->B, NULL, lv->rows, lv->buc);
        for (int c = 0; c < r->ncols; c++) bound |= 1u << r->attr[c];
    }
    uint64_t cnt = 0, sum = 0, pos = 0;
    if (rc == 0) {
        const orc_rel *p = &rels[0];
        if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads) reduction(+ : cnt, sum)
        {
            orc_walk w = base;
            w.cnt = w.sum = 0;
            w.tuples = tuples;
            w.cap = cap;
            w.pos = &pos;
            int32_t iRes[ORC_MAX_ATTRS];
#pragma omp for schedule(dynamic, 256)
            for (int64_t i = 0; i < (int64_t)p->n; i++) {
                memset(iRes, 0, sizeof(iRes));
                for (int c = 0; c < p->ncols; c++) iRes[p->attr[c]] = p->col[c][i];
                orc_dfs(&w, 0, iRes);
            }
            cnt += w.cnt;
            sum += w.sum;
        }
    }
    for (int l = 0; l < base.L; l++) {
        free(base.lv[l].buc);
        free(base.lv[l].rows);
    }
    *count = cnt;
    *checksum = sum;
    return rc;
}

/* ------------------------------------------------------------- triangle -- */

typedef struct {
    uint64_t n, len0;
    int32_t *data0, *data1;
    uint64_t *off0;
} orc_csr;

static int csr_build(const int32_t *src, const int32_t *dst, uint64_t n, orc_csr *g) {
    g->n = n;
    g->data0 = (int32_t *)malloc((n ? n : 1) * sizeof(int32_t));
    g->data1 = (int32_t *)malloc((n ? n : 1) * sizeof(int32_t));
    g->off0 = (uint64_t *)malloc((n + 1) * sizeof(uint64_t));
    if (!g->data0 || !g->data1 || !g->off0) return -2;
    return orc_trie_build(src, dst, n, g->data0, g->off0, g->data1, &g->len0);
}
static void csr_free(orc_csr *g) {
    free(g->data0);
    free(g->data1);
    free(g->off0);
}
static void csr_children(const orc_csr *g, int32_t v, uint64_t *s, uint64_t *e) {
    uint64_t lo = 0, hi = g->len0;
    while (lo < hi) {
        uint64_t mid = (lo + hi) / 2;
        if (g->data0[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    if (lo < g->len0 && g->data0[lo] == v) {
        *s = g->off0[lo];
        *e = g->off0[lo + 1];
    } else {
        *s = *e = 0;
    }
}

/* Bag semantics: every row (a,b) of R, every row (b,c) of S, every row (a,c)
 * of T.  The rows of R are walked in sorted order (the bag is unchanged). */
int orc_triangle(const int32_t *src, const int32_t *dst, uint64_t n, int nthreads, uint64_t *count,
                 uint64_t *checksum, int32_t *const *tuples, uint64_t cap) {
    orc_csr g;
    int rc = csr_build(src, dst, n, &g);
    uint64_t cnt = 0, sum = 0, pos = 0;
    if (rc == 0) {
        if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 64) reduction(+ : cnt, sum)
        for (int64_t j = 0; j < (int64_t)n; j++) {
            /* a = level-0 value owning entry j */
            uint64_t lo = 0, hi = g.len0;
            while (hi - lo > 1) {
                uint64_t mid = (lo + hi) / 2;
                if (g.off0[mid] <= (uint64_t)j) lo = mid;
                else hi = mid;
            }
            const int32_t a = g.data0[lo], b = g.data1[j];
            uint64_t sb, eb, sa = g.off0[lo], ea = g.off0[lo + 1];
            csr_children(&g, b, &sb, &eb);
            const uint64_t hab = amj_hash_step(amj_hash_step(AMJ_CHECKSUM_SEED, a), b);
            uint64_t p = sb, q = sa;
            while (p < eb && q < ea) {
                int32_t x = g.data1[p], y = g.data1[q];
                if (x < y) p++;
                else if (y < x) q++;
                else {
                    uint64_t ms = 0, mt = 0;
                    while (p < eb && g.data1[p] == x) { p++; ms++; }
                    while (q < ea && g.data1[q] == x) { q++; mt++; }
                    const uint64_t m = ms * mt;
                    cnt += m;
                    sum += m * amj_hash_step(hab, x);
                    if (tuples)
                        for (uint64_t r = 0; r < m; r++) {
                            uint64_t t;
#pragma omp atomic capture
                            t = pos++;
                            if (t < cap) {
                                tuples[0][t] = a;
                                tuples[1][t] = b;
                                tuples[2][t] = x;
                            }
                        }
                }
            }
        }
    }
    csr_free(&g);
    *count = cnt;
    *checksum = sum;
    return rc;
}

/* 4-cliques a<b<c<d of a set of oriented edges (u<v): the FOUR pattern
 * A(0,1) B(1,2) C(2,3) D(0,3) E(0,2) F(1,3) over such a relation. */
int orc_four_clique(const int32_t *src, const int32_t *dst, uint64_t n, int nthreads, uint64_t *count,
                    uint64_t *checksum) {
    orc_csr g;
    int rc = csr_build(src, dst, n, &g);
    uint64_t cnt = 0, sum = 0;
    if (rc == 0) {
        if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads) reduction(+ : cnt, sum)
        {
            int32_t *x = NULL;
            uint64_t xcap = 0;
#pragma omp for schedule(dynamic, 64)
            for (int64_t j = 0; j < (int64_t)n; j++) {
                uint64_t lo = 0, hi = g.len0;
                while (hi - lo > 1) {
                    uint64_t mid = (lo + hi) / 2;
                    if (g.off0[mid] <= (uint64_t)j) lo = mid;
                    else hi = mid;
                }
                const int32_t a = g.data0[lo], b = g.data1[j];
                uint64_t sb, eb, sa = g.off0[lo], ea = g.off0[lo + 1];
                csr_children(&g, b, &sb, &eb);
                uint64_t need = eb - sb;
                if (need > xcap) {
                    free(x);
                    xcap = need;
                    x = (int32_t *)malloc(xcap * sizeof(int32_t));
                }
                uint64_t nx = 0, p = sb, q = sa;
                while (p < eb && q < ea) {
                    int32_t u = g.data1[p], v = g.data1[q];
                    if (u < v) p++;
                    else if (v < u) q++;
                    else { x[nx++] = u; p++; q++; }
                }
                const uint64_t hab = amj_hash_step(amj_hash_step(AMJ_CHECKSUM_SEED, a), b);
                for (uint64_t i = 0; i < nx; i++) {
                    const int32_t c = x[i];
                    uint64_t sc, ec;
                    csr_children(&g, c, &sc, &ec);
                    const uint64_t habc = amj_hash_step(hab, c);
                    uint64_t r = i + 1, t = sc;
                    while (r < nx && t < ec) {
                        int32_t u = x[r], v = g.data1[t];
                        if (u < v) r++;
                        else if (v < u) t++;
                        else {
                            cnt++;
                            sum += amj_hash_step(habc, u);
                            r++;
                            t++;
                        }
                    }
                }
            }
            free(x);
        }
    }
    csr_free(&g);
    *count = cnt;
    *checksum = sum;
    return rc;
}
