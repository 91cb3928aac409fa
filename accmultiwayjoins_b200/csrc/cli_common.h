// Helpers shared by the exec-AMHJ / exec-LFTJ drivers.
#pragma once
#include <dirent.h>
#include <sys/stat.h>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include "amj.h"

namespace cli {

inline std::vector<std::string> list_files(const std::string &dir, const std::string &suffix) {
    std::vector<std::string> out;
    DIR *d = opendir(dir.c_str());
    if (!d) return out;
    while (dirent *e = readdir(d)) {
        std::string n = e->d_name;
        if (n.size() > suffix.size() && n.compare(n.size() - suffix.size(), suffix.size(), suffix) == 0) out.push_back(n);
    }
    closedir(d);
    std::sort(out.begin(), out.end());
    return out;
}

inline bool is_dir(const std::string &p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

inline int die(int rc, const char *what) {
    std::fprintf(stderr, "error: %s: %s (status %d)\n", what, amj_last_error(), rc);
    return 1;
}

// Load a .db file (schema from its name) into a device relation.
inline int load_db(amj_ctx *ctx, const std::string &path, int where, amj_rel **out,
                   std::vector<std::vector<int32_t>> &keep) {
    uint64_t n = 0;
    int ncols = 0;
    uint32_t attrs[AMJ_MAX_COLS];
    int rc = amj_db_parse_name(path.c_str(), &n, &ncols, attrs);
    if (rc) return rc;
    keep.assign(ncols, std::vector<int32_t>(n));
    std::vector<int32_t *> cols(ncols);
    for (int c = 0; c < ncols; c++) cols[c] = keep[c].data();
    rc = amj_db_read(path.c_str(), n, ncols, cols.data());
    if (rc) return rc;
    std::vector<const int32_t *> cc(cols.begin(), cols.end());
    return amj_rel_create(ctx, n, ncols, attrs, cc.data(), where, out);
}

inline void print_result(const char *op, const amj_result &r) {
    std::printf("{\"op\": \"%s\", \"count\": %llu, \"checksum\": \"%016llx\", \"build_ms\": %.3f, "
                "\"probe_ms\": %.3f, \"total_ms\": %.3f, \"tuples_per_s\": %.4g}\n",
                op, (unsigned long long)r.count, (unsigned long long)r.checksum, r.build_ms, r.probe_ms, r.total_ms,
                r.total_ms > 0 ? (double)r.count / (r.total_ms * 1e-3) : 0.0);
}

}  // namespace cli
