// exec-AMHJ <NORMAL|TRI|FOUR> <path> <ooc> <ws> <dro> <fib> [--order i,j,..] [--layout bucket|oa|cuckoo]
//           [--materialize]
// Same positional switches as the reference driver (MHJ-GPU/exec_AMHJ.cu:215-246).
// NORMAL reads every .db file of <path>; the reference asks for each file's
// position in the query on stdin (MHJ-GPU/QueryProcessor.cuh:62-63): here
// --order gives the query position of each file in name order, otherwise
// positions are read from stdin when it is not a terminal, otherwise name
// order is the query order.  TRI and FOUR read one 2-column edge file.
#include <unistd.h>
#include <cstring>
#include <sstream>
#include "cli_common.h"

int main(int argc, char **argv) {
    if (argc < 7) {
        std::fprintf(stderr, "usage: %s <NORMAL|TRI|FOUR> <path> <ooc> <ws> <dro> <fib> [--order i,j,..] "
                             "[--layout bucket|oa|cuckoo] [--materialize]\n", argv[0]);
        return 2;
    }
    std::string qt = argv[1], path = argv[2];
    const int ooc = std::atoi(argv[3]), ws = std::atoi(argv[4]), dro = std::atoi(argv[5]), fib = std::atoi(argv[6]);
    int qtype = qt == "NORMAL" ? AMJ_QUERY_NORMAL : qt == "TRI" ? AMJ_QUERY_TRI : qt == "FOUR" ? AMJ_QUERY_FOUR : -1;
    if (qtype < 0) {
        std::fprintf(stderr, "error: wrong query type %s\n", qt.c_str());
        return 2;
    }
    std::vector<int> order;
    amj_opts opts;
    std::memset(&opts, 0, sizeof(opts));
    int flags = 0;
    for (int i = 7; i < argc; i++) {
        std::string a = argv[i];
        if (a == "--order" && i + 1 < argc) {
            std::stringstream ss(argv[++i]);
            std::string t;
            while (std::getline(ss, t, ',')) order.push_back(std::atoi(t.c_str()));
        } else if (a == "--layout" && i + 1 < argc) {
            std::string l = argv[++i];
            opts.layout = l == "oa" ? AMJ_LAYOUT_OPEN_ADDR : l == "cuckoo" ? AMJ_LAYOUT_CUCKOO : AMJ_LAYOUT_BUCKET;
        } else if (a == "--materialize") {
            flags |= AMJ_F_MATERIALIZE;
        }
    }
    amj_ctx *ctx = nullptr;
    int rc = amj_ctx_create(0, &opts, &ctx);
    if (rc) return cli::die(rc, "context");
    std::vector<std::string> files;
    if (qtype == AMJ_QUERY_NORMAL) {
        if (!cli::is_dir(path)) return cli::die(AMJ_EINVAL, "NORMAL expects a directory of .db files");
        for (auto &f : cli::list_files(path, ".db")) files.push_back(path + "/" + f);
        if (files.empty()) {
            std::fprintf(stderr, "error: the directory is empty\n");
            return 1;
        }
        if (order.empty() && !isatty(0)) {
            for (size_t i = 0; i < files.size(); i++) {
                int v;
                if (std::scanf("%d", &v) != 1) break;
                order.push_back(v);
            }
            if (order.size() != files.size()) order.clear();
        }
        if (order.empty())
            for (size_t i = 0; i < files.size(); i++) order.push_back((int)i);
        if (order.size() != files.size()) return cli::die(AMJ_EINVAL, "--order needs one position per file");
    } else {
        files.push_back(path);
        order.push_back(0);
    }
    const int where = ooc ? AMJ_MEM_HOST_STREAMED : AMJ_MEM_HOST;
    std::vector<amj_rel *> rels(files.size(), nullptr);
    std::vector<std::vector<std::vector<int32_t>>> keep(files.size());
    for (size_t i = 0; i < files.size(); i++) {
        if (order[i] < 0 || (size_t)order[i] >= files.size() || rels[order[i]])
            return cli::die(AMJ_EINVAL, "bad table order");
        const int w = (ooc && order[i] == 0) ? where : AMJ_MEM_HOST;
        rc = cli::load_db(ctx, files[i], w, &rels[order[i]], keep[i]);
        if (rc) return cli::die(rc, files[i].c_str());
    }
    amj_result res;
    rc = amj_amhj_execute(ctx, qtype, rels.data(), (int)rels.size(), ooc, ws, dro, fib, flags, &res);
    if (rc) return cli::die(rc, "amhj_execute");
    cli::print_result("AMHJ", res);
    amj_result_release(&res);
    for (auto *r : rels) amj_rel_release(r);
    amj_ctx_destroy(ctx);
    return 0;
}
