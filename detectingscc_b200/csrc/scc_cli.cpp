// The `scc` command line, a drop-in for the reference's ./scc (scc.cu:21-115):
//
//   scc -a [g/h/x/y] -p [0/1] -q [0/1] -w [1/2/4/8/16/32] -f <file>
//
// Same option letters and defaults (trim1 = trim2 = true, w = 1,
// scc.cu:30-31), the same "at least 11 arguments" rule and help text
// (scc.cu:8-26), the same stdout (via the vHong / vSlota / wHong / wSlota
// shims), the same catch of the out-of-memory message (scc.cu:104-108) and
// the trailing newline (scc.cu:109).  Differences: -a d (detectSCC, the
// METIS-partitioned experiment) is not provided and is reported as an
// error; an invalid -w is rejected instead of silently skipping the BFS;
// an unreadable graph exits with status 1.
//
// Extra long options (after the required ones):
//   --labels FILE   write the canonical labels (V uint32, little-endian)
//   --json          print one JSON line with counts and timings to stderr
#include <getopt.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/scc_compat.h"
#include "scc_host.h"

static void print_help()
{
    printf("To execute:\n");
    printf("./scc -a [g/h/x/y/d] -p [0/1] -q [0/1] -w [1/2/4/8/16/32] -f <file>\n");
    printf("-a algorith to use   g - vHong, h - vSlota, x - wHong, y - wSlota, d - detectSCC\n");
    printf("-p Trim-1 enable\n");
    printf("-q Trim-2 enable\n");
    printf("-w warp size\n");
    printf("-f input file\n");
    printf("Please note that the input graph must be in GTgraph format\n");
    printf("If not provided the results are undefined\n");
}

int main(int argc, char **argv)
{
    if (argc < 11) {
        print_help();
        return 1;
    }
    const char *file = nullptr, *labels_path = nullptr;
    char algo = 0;
    bool trim1 = true, trim2 = true, json = false;
    int warpSize = 1;
    static struct option longopts[] = {{"labels", required_argument, nullptr, 'L'},
                                       {"json", no_argument, nullptr, 'J'},
                                       {nullptr, 0, nullptr, 0}};
    int c;
    while ((c = getopt_long(argc, argv, "a:p:q:w:f:", longopts, nullptr)) != -1) {
        switch (c) {
        case 'a': algo = optarg[0]; break;
        case 'p': trim1 = optarg[0] == '0' ? false : true; break;
        case 'q': trim2 = optarg[0] == '0' ? false : true; break;
        case 'w': warpSize = atoi(optarg); break;
        case 'f': file = optarg; break;
        case 'L': labels_path = optarg; break;
        case 'J': json = true; break;
        default: print_help(); return 1;
        }
    }
    if (algo != 'g' && algo != 'h' && algo != 'x' && algo != 'y' && algo != 'd') {
        print_help();
        return 1;
    }
    if ((algo == 'x' || algo == 'y') &&
        !(warpSize == 1 || warpSize == 2 || warpSize == 4 || warpSize == 8 || warpSize == 16 || warpSize == 32)) {
        fprintf(stderr, "scc: -w must be one of 1, 2, 4, 8, 16, 32\n");
        return 1;
    }
    uint32_t CSize = 0, RSize = 0;
    uint32_t *Fc = nullptr, *Fr = nullptr, *Bc = nullptr, *Br = nullptr, *Pr = nullptr;
    loadFullGraph(file ? file : "", &CSize, &RSize, &Fc, &Fr, &Bc, &Br, &Pr);
    if (!Fr) return 1;

    try {
        switch (algo) {
        case 'g': vHong(CSize, RSize, Fc, Fr, Bc, Br, trim1, trim2); break;
        case 'h': vSlota(CSize, RSize, Fc, Fr, Bc, Br, trim1, trim2); break;
        case 'x': wHong(CSize, RSize, Fc, Fr, Bc, Br, trim1, trim2, warpSize); break;
        case 'y': wSlota(CSize, RSize, Fc, Fr, Bc, Br, trim1, trim2, warpSize); break;
        case 'd': detectSCC(CSize, RSize, Fc, Fr, Bc, Br, Pr, trim1, trim2); break;
        }
    } catch (const char *e) {
        printf("%s\n", e);
        return 1;
    }
    printf("\n");
    fflush(stdout);

    if ((labels_path || json) && algo != 'd') {
        scc_context *ctx = nullptr;
        int rc = scc_create(getenv("SCC_DEVICE") ? atoi(getenv("SCC_DEVICE")) : 0, &ctx);
        uint32_t *labels = labels_path ? new uint32_t[RSize ? RSize : 1] : nullptr;
        scc_stats st;
        if (rc == SCC_OK) {
            scc_csr_view g{RSize, CSize, Fr, Fc, Br, Bc};
            rc = scc_run(ctx, &g, algo, (trim1 ? SCC_FLAG_TRIM1 : 0u) | (trim2 ? SCC_FLAG_TRIM2 : 0u), warpSize,
                         labels, &st, nullptr);
        }
        if (rc != SCC_OK) {
            fprintf(stderr, "scc: %s\n", scc_status_string(rc));
            return 1;
        }
        if (labels_path) {
            FILE *f = fopen(labels_path, "wb");
            if (!f || fwrite(labels, 4, RSize, f) != RSize) {
                fprintf(stderr, "scc: cannot write %s\n", labels_path);
                return 1;
            }
            fclose(f);
        }
        if (json)
            fprintf(stderr,
                    "{\"algo\": \"%c\", \"V\": %u, \"E\": %u, \"num_sccs\": %llu, \"num_trim1\": %llu, "
                    "\"num_trim2\": %llu, \"num_pivot\": %llu, \"passes\": %u, \"outer_iters\": %u, "
                    "\"kernel_ms\": %.4f, \"total_ms\": %.4f}\n",
                    algo, RSize, CSize, (unsigned long long)st.num_sccs, (unsigned long long)st.num_trim1,
                    (unsigned long long)st.num_trim2, (unsigned long long)st.num_pivot, st.passes, st.outer_iters,
                    st.kernel_ms, st.total_ms);
        delete[] labels;
        scc_destroy(ctx);
    }
    delete[] Fr;
    delete[] Fc;
    delete[] Br;
    delete[] Bc;
    delete[] Pr;
    return 0;
}
