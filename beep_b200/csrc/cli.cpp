// cli.cpp — command-line drop-in for the reference's sgm/sgc entry point
// (src/main.cu:27-344, flags from include/Config.h:336-429):
//   beep -g <data.bel> -t <query.mtx> -m sgm|sgc [-d <device>]
// prints the reference's result line "------------- Counter = N"
// (subgraph_matching/subgraph_matching.cuh:1277) and its timing lines;
//   beep -m txt-bel|mtx-bel|tsv-bel|tsv-mtx|bel-mtx -g <src> -r <dst>
// converts a graph file as the reference does (src/main.cu:40-67). The
// converters need no GPU.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include <unistd.h>

#include "../../include/beep.h"

namespace {

void usage(const char *argv0) {
    std::printf("Usage:  %s [options]\n\n"
                "Options:\n"
                "    -g <Src graph FileName>       data graph (.bel); the input file of a conversion\n"
                "    -r <Dst graph FileName>       the output file of a conversion\n"
                "    -t <Pattern graph filename>   query graph (.mtx, 0-based, both directions)\n"
                "    -m <MainTask>                 sgm (enumeration count) or sgc (counting), or a converter:\n"
                "                                  txt-bel, mtx-bel, tsv-bel, tsv-mtx, bel-mtx\n"
                "    -d <Device Id>                GPU device id (default = 0)\n"
                "    -s                            accepted for compatibility (edges are always sorted)\n"
                "    -c <cutoff>                   accepted for compatibility (recomputed from the degrees)\n"
                "    -h                            help\n",
                argv0);
}

int die(const char *what, beep_status s) {
    char buf[1024];
    beep_last_error(buf, sizeof(buf));
    std::fprintf(stderr, "%s failed: %s (%s)\n", what, beep_status_string(s), buf);
    return 1;
}

} // namespace

int main(int argc, char **argv) {
    const char *gpath = nullptr, *tpath = nullptr, *rpath = nullptr, *mode_s = "sgm";
    int dev = 0;
    int opt;
    while ((opt = getopt(argc, argv, "g:r:t:m:d:sc:n:h")) != -1) {
        switch (opt) {
        case 'g':
            gpath = optarg;
            break;
        case 'r':
            rpath = optarg;
            break;
        case 't':
            tpath = optarg;
            break;
        case 'm':
            mode_s = optarg;
            break;
        case 'd':
            dev = std::atoi(optarg);
            break;
        case 's':
        case 'c':
            break;
        case 'n':
            if (std::atoi(optarg) != 1) {
                std::fprintf(stderr, "only one device per process is supported (-n 1)\n");
                return 1;
            }
            break;
        case 'h':
        default:
            usage(argv[0]);
            return opt == 'h' ? 0 : 1;
        }
    }
    static const struct {
        const char *name;
        beep_convert_task task;
    } convs[] = {{"txt-bel", BEEP_CONV_TXT_BEL},
                 {"mtx-bel", BEEP_CONV_MTX_BEL},
                 {"tsv-bel", BEEP_CONV_TSV_BEL},
                 {"tsv-mtx", BEEP_CONV_TSV_MTX},
                 {"bel-mtx", BEEP_CONV_BEL_MTX}};
    for (const auto &c : convs)
        if (std::strcmp(mode_s, c.name) == 0) {
            if (!gpath || !rpath) {
                usage(argv[0]);
                return 1;
            }
            uint64_t written = 0;
            beep_status s = beep_convert(c.task, gpath, rpath, &written);
            if (s)
                return die(c.name, s);
            std::printf("%s: %llu records written to %s\n", c.name, (unsigned long long)written, rpath);
            return 0;
        }
    beep_mode mode;
    if (std::strcmp(mode_s, "sgm") == 0)
        mode = BEEP_MODE_SGM;
    else if (std::strcmp(mode_s, "sgc") == 0)
        mode = BEEP_MODE_SGC;
    else {
        std::fprintf(stderr, "Unrecognized -mt option (Main TASK): %s\n", mode_s);
        return 1;
    }
    if (!gpath || !tpath) {
        usage(argv[0]);
        return 1;
    }
    beep_ctx *ctx = nullptr;
    beep_status s = beep_ctx_create(dev, nullptr, &ctx);
    if (s)
        return die("beep_ctx_create", s);
    auto t0 = std::chrono::steady_clock::now();
    beep_graph *g = nullptr;
    if ((s = beep_graph_load_bel(ctx, gpath, &g)))
        return die("beep_graph_load_bel", s);
    auto t1 = std::chrono::steady_clock::now();
    std::printf("Read graph time: %f s\n", std::chrono::duration<double>(t1 - t0).count());
    beep_query *q = nullptr;
    if ((s = beep_query_load_mtx(tpath, &q)))
        return die("beep_query_load_mtx", s);
    beep_stats st;
    auto t2 = std::chrono::steady_clock::now();
    if ((s = beep_count_ex(ctx, g, q, mode, BEEP_OPT_TIMING, &st)))
        return die("beep_count", s);
    auto t3 = std::chrono::steady_clock::now();
    std::printf("Preprocessing TIME: %f ms\n", st.prep_ms);
    std::printf("final count time %f s\n", std::chrono::duration<double>(t3 - t2).count());
    std::printf("------------- Counter = %llu\n", (unsigned long long)st.count);
    beep_query_destroy(q);
    beep_graph_destroy(g);
    beep_ctx_destroy(ctx);
    return 0;
}
