// bc2d — drop-in command line for ck-bc's program/bc-cuda (bc2d.c main,
// bc2d.c:673-1139), running on the B200 engine through include/bcg.h.
//
// Same options (getopt string "o:p:amhDR:Uf:n:r:S:E:N:H:", bc2d.c:752), same
// input format, same source selection (sources startv .. startv+min(N,nbfs)-1,
// degree-0 sources skipped and counted, bc2d.c:998,1016-1036), same result
// file "<prefix>_1X1_0.log" ("BC RESULTS", "ROWPP N", "NodeId\tBC_VAL", then
// "%d\t%.2f" of bc/2, bc2d.c:1057-1068) and the same stdout RESULTS block
// (bc2d.c:1070-1103).  Documented differences:
//   - -p accepts only 1x1 (the reference forces one GPU anyway, bc2d.c:839);
//   - -S/-E generate an R-MAT graph with the engine's seeded generator (the
//     reference lists them as DISABLED, bc2d.c:663-664);
//   - -H 1 prunes on the GPU and yields exact BC (the reference's quirks on
//     star centres, unreachable vertices and partial source ranges are not
//     reproduced); -H 2/3 print "REMOVED" and skip BC like the reference;
//   - a source id past N-1 ends the source range (the reference reads past
//     its arrays, bc2d.c:1018);
//   - per-source times: sources run in multi-source batches, so Max/Min/Mean
//     are the batch kernel time divided evenly over the rounds, and M-TEPS is
//     the aggregate rate (sum of component edges / kernel time / 2^20).
// Extensions (letters unused by the reference): -s <file> source list (one id
// per line), -F full-precision output ("%.17g" of bc/2), -G <spec> generator
// spec (see bcg_csr_generate), -W <1|3|6> sources per batch, -B <path> binary
// CSR cache of the -f graph (read when it exists, else written after parsing),
// -T fold whole pendant trees instead of one degree-1 layer (implies -H 1;
// BCG_PRUNE_TREES).
#include <getopt.h>
#include <sys/time.h>

#include <cinttypes>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "bcg.h"

static double now_us() {
    struct timeval t;
    gettimeofday(&t, nullptr);
    return t.tv_sec * 1e6 + t.tv_usec;
}

[[noreturn]] static void prexit(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    exit(EXIT_FAILURE);
}

[[noreturn]] static void usage(const char *pname) {
    prexit("Usage (BC-1GPU):\n"
           "\t %s -p 1x1 [-o outfile] [-D] [-d] [-m] [-N <# of searches>]\n"
           "\t -> to visit a graph read from file:\n"
           "\t\t -f <graph file> -n <# vertices> [-r <start vert>]\n"
           "\t -> to visit an RMAT graph:\n"
           "\t\t -S <scale> [-E <edge factor>]\n"
           "\t Where:\n"
           "\t\t -D to ENABLE debug information\n"
           "\t\t -m to DISABLE mono GPU optimization\n"
           "\t\t -U DO NOT make graph Undirected\n"
           "\t\t -H <0|1> 1-degree reduction heuristic\n"
           "\t Extensions:\n"
           "\t\t -s <file> list of source vertices (one id per line)\n"
           "\t\t -F write bc/2 with full precision (%%.17g)\n"
           "\t\t -G <spec> generate a graph (rmat:/er:/grid: spec)\n"
           "\t\t -B <path> binary CSR cache of the -f graph (read if present, else written)\n"
           "\t\t -W <1|3|6> sources per batch\n"
           "\t\t -T fold whole pendant trees (iterated 1-degree reduction; implies -H 1)\n"
           "\n",
           pname);
}

static void die_bcg(int rc, const char *what) {
    prexit("%s failed (%d): %s\n", what, rc, bcg_last_error());
}

int main(int argc, char *argv[]) {
    if (argc == 1) usage(argv[0]);
    int gread = -1;
    int scale = 21, edgef = 16;
    int debug = 0, heuristic = 0, undirected = 1, random_root = 0, mono = 1, full = 0, trees = 0;
    int R = 0, C = 0, rootset = 0;
    uint32_t width = 0;
    uint64_t N = 0, startv = 0;
    int64_t nbfs = 1;
    std::string gfile, ofile, srcfile, genspec, cachefile;

    std::string cmdline = "MPI Tasks 0\n";
    for (int i = 0; i < argc; ++i) { cmdline += " "; cmdline += argv[i]; }
    fprintf(stdout, "%s\n\n", cmdline.c_str());

    int opt;
    while ((opt = getopt(argc, argv, "o:p:amhDR:Uf:n:r:S:E:N:H:s:FG:W:B:T")) != EOF) {
#define CHECKRTYPE(exitval, o)                                        \
    {                                                                 \
        if ((exitval) == gread) prexit("Unexpected option -%c!\n", o); \
        else gread = !(exitval);                                      \
    }
        switch ((char)opt) {
            case 'H':
                if (0 == sscanf(optarg, "%d", &heuristic)) prexit("Invalid Heuristic Option (-H): %s\n", optarg);
                break;
            case 'T': trees = 1; break;
            case 'o': ofile = optarg; break;
            case 'p': {
                char buf[64];
                snprintf(buf, sizeof(buf), "%s", optarg);
                char *p = strtok(buf, "x");
                if (!p) prexit("Invalid proc mesh field.\n");
                if (0 == sscanf(p, "%d", &R)) prexit("Invalid number of rows for proc mesh (-p): %s\n", p);
                p = strtok(nullptr, "x");
                if (!p) prexit("Invalid proc mesh field.\n");
                if (0 == sscanf(p, "%d", &C)) prexit("Invalid number of columns for proc mesh (-p): %s\n", p);
                break;
            }
            case 'R':
                sscanf(optarg, "%d", &random_root);
                if (random_root != 0 && random_root != 1) prexit("Invalid random option (-R): %s\n", optarg);
                break;
            case 'D': debug = 1; break;
            case 'm': mono = 0; break;
            case 'f': CHECKRTYPE(0, 'f'); gfile = optarg; break;
            case 'n':
                CHECKRTYPE(0, 'n');
                if (0 == sscanf(optarg, "%" SCNu64, &N)) prexit("Invalid number of vertices (-n): %s\n", optarg);
                break;
            case 'r':
                if (0 == sscanf(optarg, "%" SCNu64, &startv)) prexit("Invalid root vertex (-r): %s\n", optarg);
                rootset = 1;
                break;
            case 'S':
                CHECKRTYPE(1, 'S');
                if (0 == sscanf(optarg, "%d", &scale)) prexit("Invalid scale (-S): %s\n", optarg);
                if (scale < 1 || scale > 30) prexit("Invalid scale (-S): %s\n", optarg);
                N = 1ull << scale;
                break;
            case 'E':
                CHECKRTYPE(1, 'E');
                if (0 == sscanf(optarg, "%d", &edgef)) prexit("Invalid edge factor (-S): %s\n", optarg);
                break;
            case 'N':
                if (0 == sscanf(optarg, "%" SCNd64, &nbfs)) prexit("Invalid number of bfs (-N): %s\n", optarg);
                break;
            case 'U': undirected = 0; break;
            case 's': srcfile = optarg; break;
            case 'F': full = 1; break;
            case 'G': CHECKRTYPE(1, 'G'); genspec = optarg; break;
            case 'B': cachefile = optarg; break;
            case 'W':
                if (1 != sscanf(optarg, "%u", &width)) prexit("Invalid batch width (-W): %s\n", optarg);
                break;
            case 'h':
            case '?':
            default: usage(argv[0]);
        }
#undef CHECKRTYPE
    }
    if (gread == 1) {
        if (gfile.empty() || !N)
            prexit("Graph file (-f) and number of vertices (-n) must be specified for file based bfs.\n");
    }
    if (gread == -1) prexit("Graph file (-f) and number of vertices (-n) must be specified for file based bfs.\n");
    if (0 >= R || 1024 < R || 0 >= C || 1024 < C)
        prexit("R and C must be in range [1,%d] and [1,%d], respectively.\n", 1024, 1024);
    if (R != 1 || C != 1) prexit("Only the 1x1 processor mesh is supported (-p 1x1).\n");
    if (!genspec.empty()) N = 0;  // taken from the generated graph
    if (gread == 1 && N > 0xFFFFFFFEull)
        prexit("Number of vertics per processor too big (%" PRIu64 ").\n", N);
    if (gread == 1 && startv >= N) prexit("Invalid start vertex: %" PRIu64 ".\n", startv);
    FILE *outdebug = nullptr;
    if (debug) {
        outdebug = fopen("debug_0.log", "w");
        if (!outdebug) prexit("Cannot open file %s...\n", "debug_0.log");
    }
    if (rootset > 0) random_root = 0;
    if (trees && heuristic == 0) heuristic = 1;

    fprintf(stdout, "\n\n****** DEVEL VERSION ******\n\n\n\n***************************\n\n");
    fprintf(stdout, "Total number of vertices (N): %" PRIu64 "\n", N);
    fprintf(stdout, "Processor mesh rows (R): %d\n", R);
    fprintf(stdout, "Processor mesh columns (C): %d\n", C);
    if (gread == 1) {
        fprintf(stdout, "Reading graph from file: %s\n", gfile.c_str());
    } else {
        fprintf(stdout, "RMAT graph scale: %d\n", scale);
        fprintf(stdout, "RMAT graph edge factor: %d\n", edgef);
        fprintf(stdout, "Number of bc rounds: %" PRId64 "\n", nbfs);
        if (random_root) fprintf(stdout, "Random mode\n");
        else fprintf(stdout, "First node: %" PRIu64 "\n", startv);
    }
    fprintf(stdout, "\n\n");
    if (heuristic == 0) fprintf(stdout, "HEURISTICs: OFF: %d\n", heuristic);
    else if (heuristic == 1) fprintf(stdout, "HEURISTICs: 1-degree reduction ON: %d%s\n", heuristic, trees ? " (whole pendant trees)" : "");
    fprintf(stdout, "PREFIX SCAN library: none (device-side level loop)\n");
    fprintf(stdout, "OVERLAP: ON\n");
    fprintf(stdout, "PREFIX SCAN optimization: ON\n");
    fprintf(stdout, "\n");
    if (!mono) fprintf(stdout, "MPI REMOVED\n");

    std::string resname;
    if (!ofile.empty()) {
        fprintf(stdout, "Result written to file: %s\n", ofile.c_str());
        resname = ofile + "_1X1_0.log";
    }

    // ---- graph
    bcg_host_csr g{};
    double t0 = now_us();
    int rc;
    if (gread == 1) {
        FILE *cf = cachefile.empty() ? nullptr : fopen(cachefile.c_str(), "rb");
        if (cf) {
            fclose(cf);
            rc = bcg_csr_read_binary(cachefile.c_str(), &g);
            if (rc) prexit("%s\n", bcg_last_error());
            if (g.n != N) prexit("Cache %s holds %u vertices, not N=%" PRIu64 "\n", cachefile.c_str(), g.n, N);
        } else {
            rc = bcg_csr_read_edgelist(gfile.c_str(), N, undirected, 1, &g);
            if (rc) prexit("%s\n", bcg_last_error());
            if (!cachefile.empty() && bcg_csr_write_binary(cachefile.c_str(), &g))
                fprintf(stderr, "warning: %s\n", bcg_last_error());
        }
    } else {
        std::string spec = genspec;
        if (spec.empty()) {
            char buf[256];
            snprintf(buf, sizeof(buf), "rmat:scale=%d,ef=%d,a=0.57,b=0.19,c=0.19,seed=1", scale, edgef);
            spec = buf;
        }
        rc = bcg_csr_generate(spec.c_str(), &g);
        if (rc) die_bcg(rc, "graph generation");
        N = g.n;
        if (startv >= N) prexit("Invalid start vertex: %" PRIu64 ".\n", startv);
    }
    double t1 = now_us();
    fprintf(stdout, " done in %f secs\n", (t1 - t0) / 1.0E+6);
    fprintf(stdout, "task 0 done in %f secs\n", 0.0);
    fprintf(stdout, "task 0, Creating CSC...task 0 done in %f secs\n", 0.0);

    std::vector<uint32_t> sources;
    if (!srcfile.empty()) {
        FILE *fp = fopen(srcfile.c_str(), "r");
        if (!fp) prexit("Cannot open file %s...\n", srcfile.c_str());
        uint64_t s;
        while (fscanf(fp, "%" SCNu64, &s) == 1) {
            if (s >= N) prexit("Invalid source vertex %" PRIu64 " in %s (N=%" PRIu64 ")\n", s, srcfile.c_str(), N);
            sources.push_back((uint32_t)s);
        }
        fclose(fp);
    } else {
        uint64_t nb = nbfs < 0 ? 0 : (uint64_t)nbfs;
        if (nb > N) nb = N;
        for (uint64_t ui = 0; ui < nb; ++ui) {
            uint64_t v0 = startv + ui;
            if (v0 >= N) break;
            sources.push_back((uint32_t)v0);
        }
    }

    uint32_t flags = 0;
    if (heuristic == 1) flags |= trees ? BCG_PRUNE_TREES : BCG_PRUNE_DEGREE1;
    if (!undirected) flags |= BCG_DIRECTED;
    bcg_graph *dg = nullptr;
    double tr0 = now_us();
    rc = bcg_graph_create(g.offsets, g.adj, g.n, g.nnz, flags, &dg);
    if (rc) die_bcg(rc, "bcg_graph_create");
    double tr1 = now_us();
    uint32_t pruned = 0;
    bcg_graph_info(dg, nullptr, nullptr, nullptr, &pruned);
    if (heuristic == 1) {
        fprintf(stdout, "Degree reduction graph (%d)...\n", heuristic);
        fprintf(stdout, "task 0 Total edges removed %u\n", pruned);
    }
    fprintf(stdout, "ROWBL = %" PRIu64 " - ROWPP = %" PRIu64 "\n", N, N);
    if (width) {
        rc = bcg_set_batch_width(dg, width);
        if (rc) die_bcg(rc, "bcg_set_batch_width");
    }

    fprintf(stdout, "task 0: BC computation is running...\n");
    bcg_stats st{};
    std::vector<double> bc(N, 0.0);
    uint64_t nrounds = 0, skipped = 0;
    double all_time = 0.0;
    double mteps = 0.0;
    if (heuristic > 1) {
        fprintf(stdout, "REMOVED\n");
    } else {
        rc = bcg_run(dg, sources.data(), sources.size(), &st);
        if (rc) die_bcg(rc, "bcg_run");
        nrounds = st.sources - st.skipped;
        skipped = st.skipped;
        all_time = st.kernel_ms * 1e3;  // microseconds
        if (all_time > 0) mteps = (double)st.teps_edges / (all_time / 1.0E+6) / (1024.0 * 1024.0);
        if (outdebug)
            fprintf(outdebug, "roots %" PRIu64 " batches %" PRIu64 " width %u max_depth %u visited %" PRIu64
                              " teps_edges %" PRIu64 " kernel_ms %f\n",
                    st.roots, st.batches, st.batch_width, st.max_depth, st.visited, st.teps_edges, st.kernel_ms);
    }
    double tb0 = now_us();
    rc = bcg_get_bc(dg, bc.data());
    if (rc) die_bcg(rc, "bcg_get_bc");
    double bcred_time = now_us() - tb0;

    if (!resname.empty()) {
        FILE *resout = fopen(resname.c_str(), "w");
        if (!resout) prexit("Cannot open file %s...\n", resname.c_str());
        fprintf(resout, "BC RESULTS\n");
        fprintf(resout, "ROWPP %u\n", (unsigned)N);
        fprintf(resout, "NodeId\tBC_VAL\n");
        for (uint64_t k = 0; k < N; ++k) {
            if (full) fprintf(resout, "%d\t%.17g\n", (int)k, bc[k] / 2.0);
            else fprintf(resout, "%d\t%.2f\n", (int)k, bc[k] / 2.0);
        }
        if (fclose(resout) != 0) prexit("write to %s failed\n", resname.c_str());
    }

    const double per = nrounds ? all_time / 1.0E+6 / (double)nrounds : 0.0;
    fprintf(stdout, "\n------------- RESULTS ---------------\n");
    fprintf(stdout, "ClusterId\tSkip\tRounds\tExecTime\tRoundsTime\tMax\tMin\tMean\t1-dReduTime\n");
    fprintf(stdout, "%d\t%d\t%d\t%lf\t%lf\t%lf\t%lf\t%lf\t%lf\n", 0, (int)skipped, (int)nrounds,
            (all_time + bcred_time) / 1.0E+6, all_time / 1.0E+6, per, per, per,
            heuristic == 1 ? (tr1 - tr0) / 1.0E+6 : 0.0);
    fprintf(stdout, "task 0 BC skipped: %d \n", (int)skipped);
    fprintf(stdout, "task 0 BC rounds: %d  \n", (int)nrounds);
    fprintf(stdout, "task 0 BC execution total time: %lf sec\n", (all_time + bcred_time) / 1.0E+6);
    fprintf(stdout, "task 0 BC rounds total time: %lf sec\n", all_time / 1.0E+6);
    fprintf(stdout, "task 0 BC Max time: %lf sec\n", per);
    fprintf(stdout, "task 0 BC Min time: %lf sec\n", per);
    fprintf(stdout, "task 0 BC Mean time: %lf sec\n", per);
    fprintf(stdout, "task 0 BC M-TEPS: %lf sec\n", mteps);
    if ((uint64_t)(nbfs < 0 ? 0 : nbfs) < N && srcfile.empty() && nrounds + skipped > 0) {
        const uint64_t nb = (uint64_t)nbfs;
        unsigned int vskipped = (unsigned int)((N - nb) * skipped / nb);
        fprintf(stdout, "task 0 BC simulated time: %lf sec (virtual skipped %u)\n",
                per * (double)(N - skipped - vskipped), vskipped);
    }
    if (heuristic == 1) fprintf(stdout, "task 0 1-Degree reduction: %lf sec\n", (tr1 - tr0) / 1.0E+6);
    fprintf(stdout, "\n");
    if (outdebug) fclose(outdebug);
    bcg_graph_destroy(dg);
    bcg_csr_free(&g);
    return 0;
}
