// scc_metis: the reference's METIS input converter as a command.
//
//     scc_metis GRAPH.gr [OUT.graph]
//
// The reference's tool (MetisInput.cpp:143-160) reads a GTgraph file from a
// fixed path and writes "MeTiSInput1024.graph" into the working directory
// (MetisInput.cpp:112-113).  This one takes the input path as its argument
// and writes the same layout (scc_save_metis) to OUT.graph, by default the
// reference's file name.  The loader is the library's (load.cpp semantics).
// A file that cannot be read prints the reference's message; unlike the
// reference, the exit status then is 1.
#include <cstdio>

#include "../../include/scc_b200.h"

int main(int argc, char **argv)
{
    if (argc < 2 || argc > 3) {
        printf("To execute: scc_metis GRAPH.gr [OUT.graph]\n");
        return 1;
    }
    const char *out = argc == 3 ? argv[2] : "MeTiSInput1024.graph";
    scc_host_graph g;
    int rc = scc_load_graph(argv[1], &g);
    if (rc == SCC_ERR_IO) {
        printf("Error Reading graph file\n");
        return 1;
    }
    if (rc != SCC_OK) {
        fprintf(stderr, "scc_metis: %s: %s\n", argv[1], scc_status_string(rc));
        return 1;
    }
    rc = scc_save_metis(out, &g);
    scc_free_host_graph(&g);
    if (rc != SCC_OK) {
        fprintf(stderr, "scc_metis: %s: %s\n", out, scc_status_string(rc));
        return 1;
    }
    return 0;
}
