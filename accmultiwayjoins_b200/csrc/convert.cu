// Edge-list text files to .db relations and .tr tries (host side, OpenMP).
//
// Reference converters:
//  * edgelist_2_db (MHJ-GPU/exec_el_2_db.cu:20-87): every line of a text
//    edge list holds two integers separated by any run of ' ', '|' or tab;
//    each is read with stoul and stored as int32 (so values wrap modulo
//    2^32); the two columns are written column-major to "<edgelist>.db"
//    (common-utils/file_io.h:44-67).
//  * edgelist_to_csr (LFTJ-GPU/edgelist_to_csr.cu:19-86): the same parse,
//    then the 2-level IndexedTrie of the pairs, serialised as a .tr file.
//  * switch_el.py (MHJ-GPU/switch_el.py): the same edge list with the two
//    columns swapped.
//  * tbl_2_db (MHJ-GPU/exec_tbl_2_db.cu:26-118): selected fields of a
//    delimited table (TPC-H .tbl files: fields separated by '|'; any run of
//    tab, '|' or newline separates, spaces stay inside a field), each read
//    with stoul and stored as int32, written to "<rows>_<attr>...db" with
//    the attribute ids given for the columns.
// Here one parser serves all three (swap = 1 reverses the columns).  The file
// is mapped and cut into one chunk per thread at line boundaries; each thread
// parses its lines into its own buffer, then the buffers are concatenated
// in file order.  Lines that are empty, or whose first non-separator
// character is '#' or '%' (the comment lines of SNAP and Matrix Market edge
// lists), are skipped.  A line with one token or more than two, or a token
// that is not an integer, is an error (AMJ_EINVAL, naming the line); the
// reference's parser would read past its buffers or throw on those.
#include "amj_ops.cuh"

#include <omp.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace {

inline bool is_sep(char c) { return c == ' ' || c == '|' || c == '\t' || c == '\r'; }

struct Mapped {
    const char *p = nullptr;
    size_t n = 0;
    ~Mapped() {
        if (p && n) munmap((void *)p, n);
    }
};

int map_file(const char *path, Mapped *m) {
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return amj::fail(AMJ_EIO, std::string("edgelist: cannot open ") + path);
    struct stat st;
    if (fstat(fd, &st) != 0) {
        ::close(fd);
        return amj::fail(AMJ_EIO, std::string("edgelist: stat failed for ") + path);
    }
    m->n = (size_t)st.st_size;
    if (m->n) {
        void *p = mmap(nullptr, m->n, PROT_READ, MAP_PRIVATE, fd, 0);
        if (p == MAP_FAILED) {
            ::close(fd);
            m->n = 0;
            return amj::fail(AMJ_EIO, std::string("edgelist: mmap failed for ") + path);
        }
        m->p = (const char *)p;
    }
    ::close(fd);
    return AMJ_OK;
}

// One line [s, e): 0 = skipped (blank or comment), 1 = an edge, -1 = malformed.
int parse_line(const char *s, const char *e, int32_t *u, int32_t *v) {
    int32_t val[2] = {0, 0};
    int k = 0;
    while (true) {
        while (s < e && is_sep(*s)) s++;
        if (s == e) break;
        if (k == 0 && (*s == '#' || *s == '%')) return 0;
        if (k == 2) return -1;
        bool neg = false;
        if (*s == '-' || *s == '+') {
            neg = *s == '-';
            s++;
        }
        if (s == e || *s < '0' || *s > '9') return -1;
        uint64_t x = 0;
        while (s < e && *s >= '0' && *s <= '9') x = x * 10 + (uint64_t)(*s++ - '0');
        if (s < e && !is_sep(*s)) return -1;
        // stoul then a conversion to int: the value modulo 2^32
        val[k++] = (int32_t)(uint32_t)(neg ? (0 - x) : x);
    }
    if (k == 0) return 0;
    if (k != 2) return -1;
    *u = val[0];
    *v = val[1];
    return 1;
}

// Parse the whole file into (src, dst); swap reverses the columns.
int parse_edgelist(const char *path, int swap, std::vector<int32_t> *src, std::vector<int32_t> *dst) {
    Mapped m;
    AMJ_TRY(map_file(path, &m));
    const int T = m.n < (1u << 20) ? 1 : omp_get_max_threads();
    std::vector<size_t> cut(T + 1, m.n);
    cut[0] = 0;
    for (int t = 1; t < T; t++) {
        size_t c = m.n / T * t;
        while (c < m.n && m.p[c - 1] != '\n') c++;
        cut[t] = c < cut[t - 1] ? cut[t - 1] : c;
    }
    std::vector<std::vector<int32_t>> a(T), b(T);
    std::vector<uint64_t> bad_line(T, 0);   // first malformed line of the chunk, counted from 1 within it
    std::vector<uint64_t> lines(T, 0);
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; t++) {
        const char *s = m.p + cut[t], *end = m.p + cut[t + 1];
        uint64_t ln = 0;
        while (s < end) {
            const char *nl = (const char *)memchr(s, '\n', (size_t)(end - s));
            const char *le = nl ? nl : end;
            ln++;
            int32_t u = 0, v = 0;
            const int r = parse_line(s, le, &u, &v);
            if (r < 0) {
                bad_line[t] = ln;
                break;
            }
            if (r > 0) {
                a[t].push_back(swap ? v : u);
                b[t].push_back(swap ? u : v);
            }
            s = nl ? nl + 1 : end;
        }
        lines[t] = ln;
    }
    uint64_t before = 0;
    for (int t = 0; t < T; t++) {
        if (bad_line[t])
            return amj::fail(AMJ_EINVAL, std::string("edgelist: ") + path + " line " + std::to_string(before + bad_line[t]) +
                                             ": expected two integers");
        before += lines[t];
    }
    size_t total = 0;
    for (int t = 0; t < T; t++) total += a[t].size();
    src->resize(total);
    dst->resize(total);
    size_t off = 0;
    for (int t = 0; t < T; t++) {
        if (!a[t].empty()) {
            std::memcpy(src->data() + off, a[t].data(), a[t].size() * 4);
            std::memcpy(dst->data() + off, b[t].data(), b[t].size() * 4);
        }
        off += a[t].size();
    }
    return AMJ_OK;
}

inline bool is_tbl_sep(char c) { return c == '\t' || c == '|' || c == '\n'; }

// One line [s, e) of a delimited table: the fields `want` (ascending field
// indexes, nsel of them; pos[i] = the output column of want[i]) into v.
// 0 = skipped (blank), 1 = a row, -1 = a selected field missing or not a number.
int parse_tbl_line(const char *s, const char *e, const uint32_t *want, const int *pos, int nsel, int32_t *v) {
    while (s < e && (*s == '\r' || is_tbl_sep(*s))) s++;
    if (s == e) return 0;
    uint32_t field = 0;
    int got = 0;
    while (s < e && got < nsel) {
        while (s < e && is_tbl_sep(*s)) s++;
        if (s == e) break;
        const char *t = s;
        while (t < e && !is_tbl_sep(*t)) t++;
        if (field == want[got]) {
            // stoul: leading spaces, a sign, at least one digit; the rest of the field ignored
            const char *q = s;
            while (q < t && (*q == ' ' || *q == '\r')) q++;
            bool neg = false;
            if (q < t && (*q == '-' || *q == '+')) neg = *q++ == '-';
            if (q == t || *q < '0' || *q > '9') return -1;
            uint64_t x = 0;
            while (q < t && *q >= '0' && *q <= '9') x = x * 10 + (uint64_t)(*q++ - '0');
            v[pos[got]] = (int32_t)(uint32_t)(neg ? (0 - x) : x);
            got++;
        }
        field++;
        s = t;
    }
    return got == nsel ? 1 : -1;
}

// Parse a delimited table's selected fields (fields[], in output order).
int parse_table(const char *path, const uint32_t *fields, int ncols, std::vector<std::vector<int32_t>> *cols) {
    Mapped m;
    AMJ_TRY(map_file(path, &m));
    // fields in ascending order, with their output columns
    std::vector<std::pair<uint32_t, int>> order(ncols);
    for (int c = 0; c < ncols; c++) order[c] = {fields[c], c};
    std::sort(order.begin(), order.end());
    for (int c = 1; c < ncols; c++)
        if (order[c].first == order[c - 1].first) return amj::fail(AMJ_EINVAL, "tbl_to_db: a field selected twice");
    std::vector<uint32_t> want(ncols);
    std::vector<int> pos(ncols);
    for (int c = 0; c < ncols; c++) {
        want[c] = order[c].first;
        pos[c] = order[c].second;
    }
    const int T = m.n < (1u << 20) ? 1 : omp_get_max_threads();
    std::vector<size_t> cut(T + 1, m.n);
    cut[0] = 0;
    for (int t = 1; t < T; t++) {
        size_t c = m.n / T * t;
        while (c < m.n && m.p[c - 1] != '\n') c++;
        cut[t] = c < cut[t - 1] ? cut[t - 1] : c;
    }
    std::vector<std::vector<std::vector<int32_t>>> part(T, std::vector<std::vector<int32_t>>(ncols));
    std::vector<uint64_t> bad_line(T, 0), lines(T, 0);
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; t++) {
        const char *s = m.p + cut[t], *end = m.p + cut[t + 1];
        uint64_t ln = 0;
        int32_t v[AMJ_MAX_COLS];
        while (s < end) {
            const char *nl = (const char *)memchr(s, '\n', (size_t)(end - s));
            const char *le = nl ? nl : end;
            ln++;
            const int r = parse_tbl_line(s, le, want.data(), pos.data(), ncols, v);
            if (r < 0) {
                bad_line[t] = ln;
                break;
            }
            if (r > 0)
                for (int c = 0; c < ncols; c++) part[t][c].push_back(v[c]);
            s = nl ? nl + 1 : end;
        }
        lines[t] = ln;
    }
    uint64_t before = 0;
    for (int t = 0; t < T; t++) {
        if (bad_line[t])
            return amj::fail(AMJ_EINVAL, std::string("tbl_to_db: ") + path + " line " +
                                             std::to_string(before + bad_line[t]) +
                                             ": a selected field is missing or not an integer");
        before += lines[t];
    }
    cols->assign(ncols, {});
    for (int c = 0; c < ncols; c++)
        for (int t = 0; t < T; t++) (*cols)[c].insert((*cols)[c].end(), part[t][c].begin(), part[t][c].end());
    return AMJ_OK;
}

}  // namespace

extern "C" int amj_tbl_to_db(const char *tbl_path, const uint32_t *fields, const uint32_t *attrs, int ncols,
                             const char *out_dir, char *out_path, uint64_t out_cap, uint64_t *rows) {
    if (!tbl_path || !fields || !attrs || ncols <= 0 || ncols > AMJ_MAX_COLS)
        return amj::fail(AMJ_EINVAL, "tbl_to_db: bad arguments");
    for (int c = 0; c < ncols; c++)
        if (attrs[c] >= AMJ_MAX_ATTRS) return amj::fail(AMJ_EINVAL, "tbl_to_db: attribute id >= AMJ_MAX_ATTRS");
    std::vector<std::vector<int32_t>> cols;
    AMJ_TRY(parse_table(tbl_path, fields, ncols, &cols));
    const uint64_t n = cols[0].size();
    std::string name = std::to_string(n);
    for (int c = 0; c < ncols; c++) name += "_" + std::to_string(attrs[c]);
    name += ".db";
    const std::string path = (out_dir && *out_dir) ? std::string(out_dir) + "/" + name : name;
    std::vector<const int32_t *> cp(ncols);
    for (int c = 0; c < ncols; c++) cp[c] = cols[c].data();
    AMJ_TRY(amj_db_write(path.c_str(), n, ncols, cp.data()));
    if (out_path && out_cap) {
        std::strncpy(out_path, path.c_str(), out_cap - 1);
        out_path[out_cap - 1] = 0;
    }
    if (rows) *rows = n;
    return AMJ_OK;
}

extern "C" int amj_edgelist_read(const char *path, int swap, int32_t *src, int32_t *dst, uint64_t cap,
                                 uint64_t *n) {
    if (!path || !n || (cap && (!src || !dst))) return amj::fail(AMJ_EINVAL, "edgelist_read: bad arguments");
    std::vector<int32_t> a, b;
    AMJ_TRY(parse_edgelist(path, swap, &a, &b));
    *n = a.size();
    if (cap < a.size()) {
        if (cap) return amj::fail(AMJ_EINVAL, "edgelist_read: buffers hold fewer rows than the file");
        return AMJ_OK;   // a size query
    }
    if (!a.empty()) {
        std::memcpy(src, a.data(), a.size() * 4);
        std::memcpy(dst, b.data(), b.size() * 4);
    }
    return AMJ_OK;
}

extern "C" int amj_edgelist_to_db(const char *text_path, const char *db_path, int swap, uint64_t *rows) {
    if (!text_path || !db_path) return amj::fail(AMJ_EINVAL, "edgelist_to_db: null path");
    std::vector<int32_t> a, b;
    AMJ_TRY(parse_edgelist(text_path, swap, &a, &b));
    const int32_t *cols[2] = {a.data(), b.data()};
    AMJ_TRY(amj_db_write(db_path, a.size(), 2, cols));
    if (rows) *rows = a.size();
    return AMJ_OK;
}

extern "C" int amj_edgelist_to_tr(amj_ctx *ctx, const char *text_path, const char *tr_path, int swap,
                                  uint64_t *rows) {
    if (!ctx || !text_path || !tr_path) return amj::fail(AMJ_EINVAL, "edgelist_to_tr: null argument");
    std::vector<int32_t> a, b;
    AMJ_TRY(parse_edgelist(text_path, swap, &a, &b));
    const uint32_t attrs[2] = {0, 1};
    const int32_t *cols[2] = {a.data(), b.data()};
    amj_rel *rel = nullptr;
    AMJ_TRY(amj_rel_create(ctx, a.size(), 2, attrs, cols, AMJ_MEM_HOST, &rel));
    amj_trie *t = nullptr;
    int rc = amj_trie_build(ctx, rel->d_cols[0], rel->d_cols[1], rel->n, &t);
    if (rc == AMJ_OK) rc = amj_trie_save(t, tr_path, 0, 1);
    if (t) amj_trie_release(t);
    amj_rel_release(rel);
    if (rc == AMJ_OK && rows) *rows = a.size();
    return rc;
}
