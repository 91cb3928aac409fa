// exec-tbl-2-db <table.tbl> <field0> <field1> .. <attr0> <attr1> ..
// The reference's tbl_2_db (MHJ-GPU/exec_tbl_2_db.cu:123-133): the given
// fields (0-based) of a delimited table as "<rows>_<attr0>_<attr1>...db" in
// the current directory, the columns renamed to the given attribute ids.
#include <vector>
#include "cli_common.h"

int main(int argc, char **argv) {
    if (argc < 4 || (argc % 2) != 0) {
        std::fprintf(stderr, "usage: %s <table.tbl> <field>... <attr>... (as many attributes as fields)\n", argv[0]);
        return 2;
    }
    const int n = (argc - 2) / 2;
    std::vector<uint32_t> fields, attrs;
    for (int i = 0; i < n; i++) fields.push_back((uint32_t)std::strtoul(argv[2 + i], nullptr, 10));
    for (int i = 0; i < n; i++) attrs.push_back((uint32_t)std::strtoul(argv[2 + n + i], nullptr, 10));
    char path[4096];
    uint64_t rows = 0;
    const int rc = amj_tbl_to_db(argv[1], fields.data(), attrs.data(), n, nullptr, path, sizeof(path), &rows);
    if (rc) return cli::die(rc, "tbl_to_db");
    std::printf("%llu rows written to %s\n", (unsigned long long)rows, path);
    return 0;
}
