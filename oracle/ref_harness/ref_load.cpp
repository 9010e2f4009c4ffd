// Project-written stand-in for the reference's loadFullGraph -- TEST
// INFRASTRUCTURE ONLY.  It is linked with the reference's own, unchanged
// scc.cu / scc_kernels.cu / scc_WCC.cu / scc_Coloring.cu to build the
// reference binary oracle/_ref/scc_ref that the GPU parity tests and the
// reference arm of bench.py run.
//
// Same contract as the reference loader (load.h:6, load.cpp:12-140): skip 7
// header lines, read "p sp V E", read E arcs "a u v w", sort by (u, v),
// 1-based forward CSR with Fr[0]=Fr[1]=0 and V+2 offsets, reverse CSR by
// counting sort, *oRSize = V.  Differences, all outside the SCC path:
//   * the METIS partition array Pr is read from the file named by the
//     environment variable SCC_METIS_PARTITION (one id per vertex, as
//     load.cpp:127-131 reads it) instead of the reference's hardcoded path
//     (load.cpp:115-130), and zero-filled without it; only -a d reads it;
//   * files that start with the 8-byte magic "SCCBIN01" are read as the
//     project's binary CSR (u64 V, u64 E, Fr[V+2], Fc[E], Br[V+2], Bc[E],
//     all uint32 little-endian) so large synthetic graphs skip text parsing.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <vector>
#include <algorithm>
#include <fstream>
#include <utility>

// Pr[1..V] from SCC_METIS_PARTITION when it is set; false if that file is
// unreadable or short (the reference prints its message and returns).
static bool fill_partition(uint32_t V, uint32_t *Pr)
{
    const char *path = getenv("SCC_METIS_PARTITION");
    if (!path || !*path) return true;
    std::ifstream ism(path);
    if (!ism.is_open()) return false;
    for (uint32_t k = 0; k < V; k++) {
        uint32_t x;
        if (!(ism >> x)) return false;
        Pr[k + 1] = x;
    }
    return true;
}

void loadFullGraph(const char *filename, uint32_t *oCSize, uint32_t *oRSize, uint32_t **oFc,
                   uint32_t **oFr, uint32_t **oBc, uint32_t **oBr, uint32_t **oPr)
{
    *oCSize = 0; *oRSize = 0; *oFc = *oFr = *oBc = *oBr = *oPr = nullptr;
    FILE *f = fopen(filename, "rb");
    if (!f) { printf("Error Reading graph file\n"); return; }
    char magic[8] = {0};
    size_t got = fread(magic, 1, 8, f);
    if (got == 8 && memcmp(magic, "SCCBIN01", 8) == 0) {
        uint64_t V = 0, E = 0;
        if (fread(&V, 8, 1, f) != 1 || fread(&E, 8, 1, f) != 1) { printf("Error Reading graph file\n"); fclose(f); return; }
        uint32_t *Fr = new uint32_t[V + 2], *Br = new uint32_t[V + 2];
        uint32_t *Fc = new uint32_t[E ? E : 1], *Bc = new uint32_t[E ? E : 1];
        bool ok = fread(Fr, 4, V + 2, f) == V + 2 && fread(Fc, 4, E, f) == E &&
                  fread(Br, 4, V + 2, f) == V + 2 && fread(Bc, 4, E, f) == E;
        fclose(f);
        if (!ok) { printf("Error Reading graph file\n"); return; }
        uint32_t *Pr = new uint32_t[V + 2]();
        if (!fill_partition((uint32_t)V, Pr)) { printf("Error Reading metis graph file\n"); return; }
        *oCSize = (uint32_t)E; *oRSize = (uint32_t)V;
        *oFc = Fc; *oFr = Fr; *oBc = Bc; *oBr = Br; *oPr = Pr;
        return;
    }
    fclose(f);
    std::ifstream is(filename);
    char line[256];
    for (int i = 0; i < 7; i++) is.getline(line, 256);
    char c; char tmp[256]; uint32_t V = 0, E = 0;
    is >> c >> tmp >> V >> E;
    std::vector<std::pair<int, int> > edges(E);
    for (uint32_t k = 0; k < E; k++) { uint32_t w; is >> c >> edges[k].first >> edges[k].second >> w; }
    std::sort(edges.begin(), edges.end());
    uint32_t *Fc = new uint32_t[E ? E : 1], *Fr = new uint32_t[V + 2]();
    uint32_t *Bc = new uint32_t[E ? E : 1], *Br = new uint32_t[V + 2]();
    for (uint32_t k = 0; k < E; k++) { Fr[edges[k].first + 1]++; Fc[k] = edges[k].second; }
    for (uint32_t v = 1; v < V + 2; v++) Fr[v] += Fr[v - 1];
    for (uint32_t k = 0; k < E; k++) Br[edges[k].second + 1]++;
    for (uint32_t v = 1; v < V + 2; v++) Br[v] += Br[v - 1];
    std::vector<uint32_t> fill(Br, Br + V + 2);
    for (uint32_t k = 0; k < E; k++) Bc[fill[edges[k].second]++] = (uint32_t)edges[k].first;
    uint32_t *Pr = new uint32_t[V + 2]();
    if (!fill_partition(V, Pr)) { printf("Error Reading metis graph file\n"); return; }
    *oCSize = E; *oRSize = V;
    *oFc = Fc; *oFr = Fr; *oBc = Bc; *oBr = Br; *oPr = Pr;
}
