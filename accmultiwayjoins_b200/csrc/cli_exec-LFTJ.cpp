// exec-LFTJ <path> <algo 0=BFS|1=DFS> <ooc> <ws> [--materialize] [--attr-order a,b,c]
// Same positional switches as the reference driver (LFTJ-GPU/exec_LFTJ.cu:256-268);
// --attr-order sets the binding order the reference's driver fixes to the
// identity (exec_LFTJ.cu:230-231).
// <path> is a directory: one .db file is the triangle self-join, three .db
// files a 3-relation join, two files are an error (exec_LFTJ.cu:92-95).
#include <cstring>
#include "cli_common.h"

int main(int argc, char **argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s <dir> <0=BFS|1=DFS> <ooc> <ws> [--materialize] [--attr-order a,b,..]\n",
                     argv[0]);
        return 2;
    }
    std::string path = argv[1];
    const int algo = std::atoi(argv[2]), ooc = std::atoi(argv[3]), ws = std::atoi(argv[4]);
    int flags = 0;
    std::vector<uint32_t> order;
    for (int i = 5; i < argc; i++) {
        if (std::strcmp(argv[i], "--materialize") == 0) flags |= AMJ_F_MATERIALIZE;
        else if (std::strcmp(argv[i], "--attr-order") == 0 && i + 1 < argc) {
            for (const char *p = argv[++i]; *p;) {
                char *end = nullptr;
                order.push_back((uint32_t)std::strtoul(p, &end, 10));
                if (end == p) return cli::die(AMJ_EINVAL, "--attr-order: expected a,b,c");
                p = *end == ',' ? end + 1 : end;
            }
        }
    }
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
    rc = order.empty() ? amj_lftj_execute(ctx, rels.data(), (int)rels.size(), algo, ooc, ws, flags, &res)
                       : amj_lftj_execute_ordered(ctx, rels.data(), (int)rels.size(), algo, ooc, ws, flags, order.data(),
                                                  (int)order.size(), &res);
    if (rc) return cli::die(rc, "lftj_execute");
    cli::print_result(algo == AMJ_LFTJ_DFS ? "ALFTJ-DFS" : "ALFTJ-BFS", res);
    amj_result_release(&res);
    for (auto *r : rels) amj_rel_release(r);
    amj_ctx_destroy(ctx);
    return 0;
}
