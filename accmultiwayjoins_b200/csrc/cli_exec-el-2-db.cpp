// exec-el-2-db <edgelist> [out.db] [--swap]
// The reference's edgelist_2_db (MHJ-GPU/exec_el_2_db.cu:90-96): a text edge
// list to a 2-column .db file, by default "<edgelist>.db"; --swap reverses
// the columns (MHJ-GPU/switch_el.py).
#include <cstring>
#include "cli_common.h"

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <edgelist> [out.db] [--swap]\n", argv[0]);
        return 2;
    }
    std::string in = argv[1], out;
    int swap = 0;
    for (int i = 2; i < argc; i++) {
        if (std::strcmp(argv[i], "--swap") == 0) swap = 1;
        else out = argv[i];
    }
    if (out.empty()) out = in + ".db";
    uint64_t rows = 0;
    const int rc = amj_edgelist_to_db(in.c_str(), out.c_str(), swap, &rows);
    if (rc) return cli::die(rc, "edgelist_to_db");
    std::printf("%llu rows written to %s\n", (unsigned long long)rows, out.c_str());
    return 0;
}
