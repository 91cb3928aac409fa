// edgelist-to-csr <edgelist> [out.tr] [--swap]
// The reference's edgelist_to_csr (LFTJ-GPU/edgelist_to_csr.cu:89-98): a text
// edge list to the .tr file of its 2-level trie, by default "output.tr".
#include <cstring>
#include "cli_common.h"

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <edgelist> [out.tr] [--swap]\n", argv[0]);
        return 2;
    }
    std::string in = argv[1], out = "output.tr";
    int swap = 0;
    for (int i = 2; i < argc; i++) {
        if (std::strcmp(argv[i], "--swap") == 0) swap = 1;
        else out = argv[i];
    }
    amj_ctx *ctx = nullptr;
    int rc = amj_ctx_create(0, nullptr, &ctx);
    if (rc) return cli::die(rc, "context");
    uint64_t rows = 0;
    rc = amj_edgelist_to_tr(ctx, in.c_str(), out.c_str(), swap, &rows);
    amj_ctx_destroy(ctx);
    if (rc) return cli::die(rc, "edgelist_to_tr");
    std::printf("%llu edges, trie written to %s\n", (unsigned long long)rows, out.c_str());
    return 0;
}
