// exec-LFTJ <path> <algo 0=BFS|1=DFS> <ooc> <ws> [--materialize]
// Same positional switches as the reference driver (LFTJ-GPU/exec_LFTJ.cu:256-268).
// <path> is a directory: one .db file is the triangle self-join, three .db
// files a 3-relation join, two files are an error (exec_LFTJ.cu:92-95).
#include <cstring>
#include "cli_common.h"

int main(int argc, char **argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s <dir> <0=BFS|1=DFS> <ooc> <ws> [--materialize]\n", argv[0]);
        return 2;
    }
    std::string path = argv[1];
    const int algo = std::atoi(argv[2]), ooc = std::atoi(argv[3]), ws = std::atoi(argv[4]);
    int flags = 0;
    for (int i = 5; i < argc; i++)
        if (std::strcmp(argv[i], "--materialize") == 0) flags |= AMJ_F_MATERIALIZE;
    amj_ctx *ctx = nullptr;
    int rc = amj_ctx_create(0, nullptr, &ctx);
    if (rc) return cli::die(rc, "context");
    std::vector<std::string> files;
    if (cli::is_dir(path))
        for (auto &f : cli::list_files(path, ".db")) files.push_back(path + "/" + f);
    else
        files.push_back(path);
    std::vector<amj_rel *> rels(files.size(), nullptr);
    std::vector<std::vector<std::vector<int32_t>>> keep(files.size());
    for (size_t i = 0; i < files.size(); i++) {
        rc = cli::load_db(ctx, files[i], AMJ_MEM_HOST, &rels[i], keep[i]);
        if (rc) return cli::die(rc, files[i].c_str());
    }
    amj_result res;
    rc = amj_lftj_execute(ctx, rels.data(), (int)rels.size(), algo, ooc, ws, flags, &res);
    if (rc) return cli::die(rc, "lftj_execute");
    cli::print_result(algo == AMJ_LFTJ_DFS ? "ALFTJ-DFS" : "ALFTJ-BFS", res);
    amj_result_release(&res);
    for (auto *r : rels) amj_rel_release(r);
    amj_ctx_destroy(ctx);
    return 0;
}
