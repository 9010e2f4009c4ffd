// GTgraph loader and CSR / transpose builder.
//
// Same contract as the reference loader (load.h:6, load.cpp:12-140):
//   * skip 7 header lines, read "p sp V E" (load.cpp:32-36);
//   * read exactly E arcs "a u v w", w ignored (load.cpp:42-45);
//   * order the arcs by (u, v), duplicates and self-loops kept (load.cpp:47);
//   * forward CSR, 1-based, Fr[V+2] with Fr[0] = Fr[1] = 0 (load.cpp:49-77);
//   * reverse CSR whose in-lists hold sources in ascending order
//     (load.cpp:80-113);
//   * *oRSize = V, *oCSize = E (load.cpp:133-134).
// Differences: the (u, v) order comes from two stable counting sorts
// (O(E + V)) instead of std::sort; ids outside [1, V] and short files are
// reported instead of being undefined behaviour; the METIS partition array
// Pr, which only the detectSCC driver reads, is read from the file named by
// SCC_METIS_PARTITION (zero-filled without it) instead of the reference's
// hardcoded path (load.cpp:115-130).  Files that start with "SCCBIN01" are read as the
// project's binary CSR (see scc_load_graph).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "scc_host.h"
#include "../../include/scc_compat.h"

namespace {

struct Buf {
    char *p = nullptr;
    size_t n = 0;
    ~Buf() { free(p); }
};

bool read_file(const char *path, Buf &b)
{
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    if (fseek(f, 0, SEEK_END) != 0) { fclose(f); return false; }
    long sz = ftell(f);
    if (sz < 0) { fclose(f); return false; }
    fseek(f, 0, SEEK_SET);
    b.p = (char *)malloc((size_t)sz + 1);
    if (!b.p) { fclose(f); return false; }
    b.n = fread(b.p, 1, (size_t)sz, f);
    b.p[b.n] = 0;
    fclose(f);
    return b.n == (size_t)sz;
}

inline const char *skip_ws(const char *s, const char *e)
{
    while (s < e && (*s == ' ' || *s == '\t' || *s == '\n' || *s == '\r')) s++;
    return s;
}
inline const char *skip_tok(const char *s, const char *e)
{
    while (s < e && !(*s == ' ' || *s == '\t' || *s == '\n' || *s == '\r')) s++;
    return s;
}
inline bool read_u64(const char *&s, const char *e, uint64_t &out)
{
    s = skip_ws(s, e);
    if (s >= e) return false;
    bool neg = false;
    if (*s == '-' || *s == '+') { neg = *s == '-'; s++; }
    if (s >= e || *s < '0' || *s > '9') return false;
    uint64_t x = 0;
    while (s < e && *s >= '0' && *s <= '9') { x = x * 10 + (uint64_t)(*s - '0'); s++; }
    out = neg ? (uint64_t)0 - x : x;
    return true;
}

}  // namespace

// Build forward + reverse CSR from an arc list (1-based ids already checked).
int scc_build_csr(uint32_t V, uint64_t E, const uint32_t *src, const uint32_t *dst, scc_host_graph *g)
{
    memset(g, 0, sizeof(*g));
    if (E > 0xFFFFFFFFull) return SCC_ERR_TOO_LARGE;
    const size_t nv = (size_t)V + 2, ne = E ? (size_t)E : 1;
    g->Fr = new (std::nothrow) uint32_t[nv]();
    g->Br = new (std::nothrow) uint32_t[nv]();
    g->Fc = new (std::nothrow) uint32_t[ne];
    g->Bc = new (std::nothrow) uint32_t[ne];
    g->Pr = new (std::nothrow) uint32_t[nv]();
    std::vector<uint32_t> tmp_u, tmp_v;
    try {
        tmp_u.resize(ne);
        tmp_v.resize(ne);
    } catch (...) {
        scc_free_host_graph(g);
        return SCC_ERR_OOM;
    }
    if (!g->Fr || !g->Br || !g->Fc || !g->Bc || !g->Pr) { scc_free_host_graph(g); return SCC_ERR_OOM; }
    g->V = V;
    g->E = (uint32_t)E;
    uint32_t *Fr = g->Fr, *Br = g->Br;
    // pass 1: stable counting sort by v (Br counts in-degree)
    for (uint64_t k = 0; k < E; k++) Br[dst[k] + 1]++;
    for (size_t v = 1; v < nv; v++) Br[v] += Br[v - 1];
    {
        std::vector<uint32_t> fill(Br, Br + nv);
        for (uint64_t k = 0; k < E; k++) {
            uint32_t pos = fill[dst[k]]++;
            tmp_u[pos] = src[k];
            tmp_v[pos] = dst[k];
        }
    }
    // pass 2: stable counting sort by u -> arcs in (u, v) order = Fc
    for (uint64_t k = 0; k < E; k++) Fr[src[k] + 1]++;
    for (size_t v = 1; v < nv; v++) Fr[v] += Fr[v - 1];
    {
        std::vector<uint32_t> fill(Fr, Fr + nv);
        for (uint64_t k = 0; k < E; k++) g->Fc[fill[tmp_u[k]]++] = tmp_v[k];
    }
    // reverse CSR: walk arcs in (u, v) order, append u to v's list
    // (load.cpp:103-111), so each in-list is ascending in u
    {
        std::vector<uint32_t> fill(Br, Br + nv);
        for (uint32_t u = 1; u <= V; u++)
            for (uint32_t e = Fr[u]; e < Fr[u + 1]; e++) g->Bc[fill[g->Fc[e]]++] = u;
    }
    return SCC_OK;
}

extern "C" void scc_free_host_graph(scc_host_graph *g)
{
    if (!g) return;
    delete[] g->Fr; delete[] g->Fc; delete[] g->Br; delete[] g->Bc; delete[] g->Pr;
    memset(g, 0, sizeof(*g));
}

static int load_binary(const Buf &b, scc_host_graph *g)
{
    if (b.n < 24) return SCC_ERR_BAD_GRAPH;
    uint64_t V, E;
    memcpy(&V, b.p + 8, 8);
    memcpy(&E, b.p + 16, 8);
    if (V > SCC_MAX_VERTICES || E > 0xFFFFFFFFull) return SCC_ERR_TOO_LARGE;
    size_t need = 24 + 4 * (2 * (V + 2) + 2 * E);
    if (b.n < need) return SCC_ERR_BAD_GRAPH;
    memset(g, 0, sizeof(*g));
    const size_t nv = V + 2, ne = E ? E : 1;
    g->Fr = new (std::nothrow) uint32_t[nv];
    g->Br = new (std::nothrow) uint32_t[nv];
    g->Fc = new (std::nothrow) uint32_t[ne];
    g->Bc = new (std::nothrow) uint32_t[ne];
    g->Pr = new (std::nothrow) uint32_t[nv]();
    if (!g->Fr || !g->Br || !g->Fc || !g->Bc || !g->Pr) { scc_free_host_graph(g); return SCC_ERR_OOM; }
    const char *p = b.p + 24;
    memcpy(g->Fr, p, nv * 4); p += nv * 4;
    memcpy(g->Fc, p, E * 4); p += E * 4;
    memcpy(g->Br, p, nv * 4); p += nv * 4;
    memcpy(g->Bc, p, E * 4);
    g->V = (uint32_t)V;
    g->E = (uint32_t)E;
    return SCC_OK;
}

extern "C" int scc_load_graph(const char *path, scc_host_graph *g)
{
    if (!path || !g) return SCC_ERR_INVALID_ARG;
    memset(g, 0, sizeof(*g));
    Buf b;
    if (!read_file(path, b)) return SCC_ERR_IO;
    if (b.n >= 8 && memcmp(b.p, "SCCBIN01", 8) == 0) return load_binary(b, g);
    const char *s = b.p, *e = b.p + b.n;
    // load.cpp:32-33: skip seven lines
    for (int i = 0; i < 7; i++) {
        while (s < e && *s != '\n') s++;
        if (s < e) s++;
    }
    // load.cpp:36: "p sp V E"
    s = skip_ws(s, e);
    s = skip_tok(s, e);          // 'p'
    s = skip_ws(s, e);
    s = skip_tok(s, e);          // 'sp'
    uint64_t V = 0, E = 0;
    if (!read_u64(s, e, V) || !read_u64(s, e, E)) return SCC_ERR_BAD_GRAPH;
    if (V > SCC_MAX_VERTICES) return SCC_ERR_TOO_LARGE;
    if (E > 0xFFFFFFFFull) return SCC_ERR_TOO_LARGE;
    std::vector<uint32_t> src, dst;
    try {
        src.resize(E ? E : 1);
        dst.resize(E ? E : 1);
    } catch (...) {
        return SCC_ERR_OOM;
    }
    for (uint64_t k = 0; k < E; k++) {
        // "a u v w" (load.cpp:43): one token, then three integers
        s = skip_ws(s, e);
        if (s >= e) return SCC_ERR_BAD_GRAPH;
        s++;  // the arc letter (read as a single char by the reference)
        uint64_t u, v, w;
        if (!read_u64(s, e, u) || !read_u64(s, e, v) || !read_u64(s, e, w)) return SCC_ERR_BAD_GRAPH;
        if (u < 1 || u > V || v < 1 || v > V) return SCC_ERR_BAD_GRAPH;
        src[k] = (uint32_t)u;
        dst[k] = (uint32_t)v;
    }
    return scc_build_csr((uint32_t)V, E, src.data(), dst.data(), g);
}

extern "C" int scc_save_binary(const char *path, const scc_host_graph *g)
{
    if (!path || !g) return SCC_ERR_INVALID_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return SCC_ERR_IO;
    uint64_t V = g->V, E = g->E;
    bool ok = fwrite("SCCBIN01", 1, 8, f) == 8 && fwrite(&V, 8, 1, f) == 1 && fwrite(&E, 8, 1, f) == 1 &&
              fwrite(g->Fr, 4, V + 2, f) == V + 2 && fwrite(g->Fc, 4, E, f) == E &&
              fwrite(g->Br, 4, V + 2, f) == V + 2 && fwrite(g->Bc, 4, E, f) == E;
    ok = (fclose(f) == 0) && ok;
    return ok ? SCC_OK : SCC_ERR_IO;
}

namespace {

// Appends the decimal digits of x and one space.
inline char *put_u32_sp(char *o, uint32_t x)
{
    char tmp[10];
    int n = 0;
    do {
        tmp[n++] = (char)('0' + x % 10u);
        x /= 10u;
    } while (x);
    while (n) *o++ = tmp[--n];
    *o++ = ' ';
    return o;
}

}  // namespace

// The reference converter's METIS layout (MetisInput.cpp:114-131): "V E",
// then per vertex its forward list and its reverse list.  Written through
// one buffer flushed every few MB.
extern "C" int scc_save_metis(const char *path, const scc_host_graph *g)
{
    if (!path || !g || (g->V && (!g->Fr || !g->Br)) || (g->E && (!g->Fc || !g->Bc))) return SCC_ERR_INVALID_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return SCC_ERR_IO;
    const size_t cap = 4u << 20;
    std::vector<char> buf;
    try {
        buf.resize(cap + 64);
    } catch (...) {
        fclose(f);
        return SCC_ERR_OOM;
    }
    char *o = buf.data();
    bool ok = true;
    auto flush = [&](bool force) {
        if (force || (size_t)(o - buf.data()) >= cap) {
            const size_t n = (size_t)(o - buf.data());
            ok = ok && fwrite(buf.data(), 1, n, f) == n;
            o = buf.data();
        }
    };
    o += snprintf(o, 64, "%u %u\n", g->V, g->E);
    for (uint32_t v = 1; v <= g->V; v++) {
        for (uint32_t e = g->Fr[v]; e < g->Fr[v + 1]; e++) {
            o = put_u32_sp(o, g->Fc[e]);
            flush(false);
        }
        for (uint32_t e = g->Br[v]; e < g->Br[v + 1]; e++) {
            o = put_u32_sp(o, g->Bc[e]);
            flush(false);
        }
        *o++ = '\n';
        flush(false);
    }
    flush(true);
    ok = (fclose(f) == 0) && ok;
    return ok ? SCC_OK : SCC_ERR_IO;
}

// GTgraph text: the seven comment lines the reference skips, "p sp V E",
// then "a u v 1" per arc in forward order.
extern "C" int scc_save_gtgraph(const char *path, const scc_host_graph *g)
{
    if (!path || !g || (g->V && !g->Fr) || (g->E && !g->Fc)) return SCC_ERR_INVALID_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return SCC_ERR_IO;
    const size_t cap = 4u << 20;
    std::vector<char> buf;
    try {
        buf.resize(cap + 128);
    } catch (...) {
        fclose(f);
        return SCC_ERR_OOM;
    }
    char *o = buf.data();
    bool ok = true;
    o += snprintf(o, 128, "c FILE\t\t\t: graph\nc No. of vertices\t: %u\nc No. of directed edges\t: %u\n", g->V, g->E);
    ok = ok && fwrite(buf.data(), 1, (size_t)(o - buf.data()), f) == (size_t)(o - buf.data());
    o = buf.data();
    o += snprintf(o, 128, "c Max. weight\t\t: 1\nc Min. weight\t\t: 1\nc A directed arc from u to v of weight w\n");
    o += snprintf(o, 128, "c is represented below as ' a  u  v  w '\np sp %u %u\n", g->V, g->E);
    for (uint32_t u = 1; u <= g->V; u++)
        for (uint32_t e = g->Fr[u]; e < g->Fr[u + 1]; e++) {
            *o++ = 'a';
            *o++ = ' ';
            o = put_u32_sp(o, u);
            o = put_u32_sp(o, g->Fc[e]);
            *o++ = '1';
            *o++ = '\n';
            if ((size_t)(o - buf.data()) >= cap) {
                ok = ok && fwrite(buf.data(), 1, (size_t)(o - buf.data()), f) == (size_t)(o - buf.data());
                o = buf.data();
            }
        }
    ok = ok && fwrite(buf.data(), 1, (size_t)(o - buf.data()), f) == (size_t)(o - buf.data());
    ok = (fclose(f) == 0) && ok;
    return ok ? SCC_OK : SCC_ERR_IO;
}

// One partition id per vertex, whitespace separated (load.cpp:127-131).
extern "C" int scc_load_partition(const char *path, uint32_t V, uint32_t *Pr)
{
    if (!path || !Pr) return SCC_ERR_INVALID_ARG;
    Buf b;
    if (!read_file(path, b)) return SCC_ERR_IO;
    const char *s = b.p, *e = b.p + b.n;
    Pr[0] = 0;
    Pr[V + 1] = 0;
    for (uint32_t k = 1; k <= V; k++) {
        uint64_t x = 0;
        if (!read_u64(s, e, x) || x > 0xFFFFFFFFull) return SCC_ERR_BAD_GRAPH;
        Pr[k] = (uint32_t)x;
    }
    return SCC_OK;
}

// The reference's loader signature (load.h:6).  On a read failure it prints
// the reference's message and leaves empty outputs (the reference returns
// with them unset, load.cpp:24-28).
void loadFullGraph(const char *filename, uint32_t *oCSize, uint32_t *oRSize, uint32_t **oFc, uint32_t **oFr,
                   uint32_t **oBc, uint32_t **oBr, uint32_t **oPr)
{
    scc_host_graph g;
    int rc = scc_load_graph(filename, &g);
    if (rc != SCC_OK) {
        if (rc == SCC_ERR_IO) printf("Error Reading graph file\n");
        else fprintf(stderr, "loadFullGraph: %s: %s\n", filename, scc_status_string(rc));
        *oCSize = 0;
        *oRSize = 0;
        *oFc = *oFr = *oBc = *oBr = *oPr = nullptr;
        return;
    }
    // the METIS partition that only detectSCC reads: the reference opens a
    // fixed path (load.cpp:115-130); here the path comes from the
    // environment, and its absence leaves Pr zero-filled (one partition)
    const char *part = getenv("SCC_METIS_PARTITION");
    if (part && *part && g.Pr && scc_load_partition(part, g.V, g.Pr) != SCC_OK) {
        printf("Error Reading metis graph file\n");
        scc_free_host_graph(&g);
        *oCSize = 0;
        *oRSize = 0;
        *oFc = *oFr = *oBc = *oBr = *oPr = nullptr;
        return;
    }
    *oCSize = g.E;
    *oRSize = g.V;
    *oFc = g.Fc;
    *oFr = g.Fr;
    *oBc = g.Bc;
    *oBr = g.Br;
    *oPr = g.Pr;
}

extern "C" int scc_graph_from_arcs(uint32_t V, uint64_t E, const uint32_t *src, const uint32_t *dst,
                                   scc_host_graph *out)
{
    if (!out || (E && (!src || !dst))) return SCC_ERR_INVALID_ARG;
    if (V > SCC_MAX_VERTICES) return SCC_ERR_TOO_LARGE;
    for (uint64_t k = 0; k < E; k++)
        if (src[k] < 1 || src[k] > V || dst[k] < 1 || dst[k] > V) return SCC_ERR_BAD_GRAPH;
    return scc_build_csr(V, E, src, dst, out);
}
