/*
 * CPU oracle for the SCC hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Nothing in the product (the CUDA library, the CLI, the shims) links or
 * calls this file.  Only tests/, the smoke check and bench.py's CPU-baseline
 * leg load it, and only as the checker or as the timed CPU baseline.
 *
 * Two independent oracles live here:
 *
 *   oracle_tarjan      an iterative (non-recursive) Tarjan SCC over the
 *                      forward CSR, canonicalised so every vertex carries
 *                      the minimum vertex id of its component.  Used as the
 *                      label oracle and as the timed CPU baseline.
 *
 *   oracle_hong        sequential restatements of the reference's phase
 *   oracle_slota       schedules (vHong, scc_WCC.cu:573-930; vSlota,
 *                      scc_Coloring.cu:403-637).  They reproduce the phase
 *                      order, the trim rules, the pivot rule and the
 *                      counters the reference prints (numberOf1Sccs and
 *                      Number Of Sccs), with the deterministic choices the
 *                      CUDA engine makes where the reference races:
 *                        - pivot = argmax of the uint32 product
 *                          out-degree * in-degree (scc_kernels.cu:643-656,
 *                          :57-74), ties to the smallest id;
 *                        - single-pass kernels (trim-2, vSlota's single
 *                          trim-1) decide on the state at the start of the
 *                          pass;
 *                        - every live range gets a pivot (the reference's
 *                          "newDegree > oldDegree" against vertex 0 can leave
 *                          a range without one and then loops forever).
 *
 * Graph layout is the reference's (load.cpp:49-113): 1-based vertices,
 * Fr/Br have V+2 entries with Fr[0]=Fr[1]=0, vertex v owns
 * Fc[Fr[v] .. Fr[v+1]); Bc/Br is the transpose.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_OK 0
#define OR_ERR_OOM 3

#define DEADR 0xFFFFFFFFu

/* ------------------------------------------------------------------ */
/* Tarjan                                                             */
/* ------------------------------------------------------------------ */

/* labels has V+1 entries; labels[0] is set to 0.  Returns the number of
 * SCCs, or -1 when memory runs out. */
long long oracle_tarjan(uint32_t V, const uint32_t *Fr, const uint32_t *Fc,
                        uint32_t *labels)
{
    uint32_t *index = (uint32_t *)malloc((size_t)(V + 1) * sizeof(uint32_t));
    uint32_t *low = (uint32_t *)malloc((size_t)(V + 1) * sizeof(uint32_t));
    uint32_t *stk = (uint32_t *)malloc((size_t)(V + 1) * sizeof(uint32_t));
    uint32_t *cs_v = (uint32_t *)malloc((size_t)(V + 1) * sizeof(uint32_t));
    uint32_t *cs_e = (uint32_t *)malloc((size_t)(V + 1) * sizeof(uint32_t));
    unsigned char *onstk = (unsigned char *)calloc((size_t)V + 1, 1);
    if (!index || !low || !stk || !cs_v || !cs_e || !onstk) {
        free(index); free(low); free(stk); free(cs_v); free(cs_e); free(onstk);
        return -1;
    }
    for (uint32_t v = 0; v <= V; v++) index[v] = 0; /* 0 = unvisited */
    uint32_t next_index = 1, sp = 0;
    long long nscc = 0;
    labels[0] = 0;
    for (uint32_t root = 1; root <= V; root++) {
        if (index[root]) continue;
        uint32_t csp = 0;
        cs_v[csp] = root; cs_e[csp] = Fr[root]; csp++;
        index[root] = low[root] = next_index++;
        stk[sp++] = root; onstk[root] = 1;
        while (csp) {
            uint32_t v = cs_v[csp - 1];
            uint32_t e = cs_e[csp - 1];
            uint32_t end = Fr[v + 1];
            int descended = 0;
            while (e < end) {
                uint32_t w = Fc[e++];
                if (!index[w]) {
                    cs_e[csp - 1] = e;
                    index[w] = low[w] = next_index++;
                    stk[sp++] = w; onstk[w] = 1;
                    cs_v[csp] = w; cs_e[csp] = Fr[w]; csp++;
                    descended = 1;
                    break;
                } else if (onstk[w] && index[w] < low[v]) {
                    low[v] = index[w];
                }
            }
            if (descended) continue;
            cs_e[csp - 1] = e;
            if (low[v] == index[v]) {
                /* pop the component, then label it with its minimum id */
                uint32_t top = sp, mn = v;
                do {
                    uint32_t w = stk[--sp];
                    if (w < mn) mn = w;
                    if (w == v) break;
                } while (1);
                for (uint32_t i = sp; i < top; i++) {
                    onstk[stk[i]] = 0;
                    labels[stk[i]] = mn;
                }
                nscc++;
            }
            csp--;
            if (csp) {
                uint32_t u = cs_v[csp - 1];
                if (low[v] < low[u]) low[u] = low[v];
            }
        }
    }
    free(index); free(low); free(stk); free(cs_v); free(cs_e); free(onstk);
    return nscc;
}

/* ------------------------------------------------------------------ */
/* Shared helpers for the phase restatements                          */
/* ------------------------------------------------------------------ */

typedef struct {
    uint32_t V;
    const uint32_t *Fr, *Fc, *Br, *Bc;
    uint32_t *range;   /* range / colour name, DEADR once assigned to an SCC */
    uint32_t *label;   /* representative id of the SCC a dead vertex is in */
    unsigned char *fv, *bv;
    uint32_t *queue;
    uint32_t *vals;    /* per-range scratch */
    uint64_t counts[3]; /* trim1 vertices, trim2 pairs, pivots */
} OState;

static inline int live(const OState *s, uint32_t x) { return s->range[x] != DEADR; }

/* uint32 product of full-graph degrees (scc_kernels.cu:651-652). */
static inline uint32_t deg_product(const OState *s, uint32_t v)
{
    return (s->Fr[v + 1] - s->Fr[v]) * (s->Br[v + 1] - s->Br[v]);
}

/* Pivot key: larger product wins, ties go to the smaller id. */
static inline uint64_t pivot_key(const OState *s, uint32_t v)
{
    return ((uint64_t)deg_product(s, v) << 32) | (uint64_t)(0xFFFFFFFFu - v);
}

/* Does v have a live neighbour in its own range in adjacency (R, C)?
 * Follows the early-exit scans of trim1 (scc_kernels.cu:197-222). */
static int has_live_same(const OState *s, const uint32_t *R, const uint32_t *C,
                         uint32_t v)
{
    uint32_t r = s->range[v];
    for (uint32_t e = R[v]; e < R[v + 1]; e++) {
        uint32_t w = C[e];
        if (s->range[w] == r) return 1;
    }
    return 0;
}

/* trim1 iterated to its fixpoint (scc_WCC.cu:680-687): a vertex without a
 * live same-range in-neighbour or out-neighbour is an SCC of its own.  The
 * fixpoint does not depend on visiting order. */
static void trim1_fixpoint(OState *s)
{
    int changed = 1;
    while (changed) {
        changed = 0;
        for (uint32_t v = 1; v <= s->V; v++) {
            if (!live(s, v)) continue;
            if (!has_live_same(s, s->Br, s->Bc, v) || !has_live_same(s, s->Fr, s->Fc, v)) {
                s->range[v] = DEADR;
                s->label[v] = v;
                s->counts[0]++;
                changed = 1;
            }
        }
    }
}

/* One trim1 pass that decides every vertex on the state before the pass
 * (vSlota runs trim1 once, scc_Coloring.cu:507-508). */
static int trim1_single_pass(OState *s)
{
    uint32_t n = 0;
    for (uint32_t v = 1; v <= s->V; v++) {
        if (!live(s, v)) continue;
        if (!has_live_same(s, s->Br, s->Bc, v) || !has_live_same(s, s->Fr, s->Fc, v))
            s->queue[n++] = v;
    }
    for (uint32_t i = 0; i < n; i++) {
        uint32_t v = s->queue[i];
        s->range[v] = DEADR;
        s->label[v] = v;
    }
    s->counts[0] += n;
    return 0;
}

/* Count live same-range neighbours of x in (R, C), stopping at 2, and
 * return the first one in *first (scc_kernels.cu:250-261). */
static uint32_t count_live_upto2(const OState *s, const uint32_t *R, const uint32_t *C,
                                 uint32_t x, uint32_t r, uint32_t *first)
{
    uint32_t n = 0;
    for (uint32_t e = R[x]; e < R[x + 1]; e++) {
        uint32_t w = C[e];
        if (s->range[w] == r) {
            n++;
            if (n == 2) break;
            if (first) *first = w;
        }
    }
    return n;
}

/* Decide trim2 for v (scc_kernels.cu:236-348).  Returns the partner k
 * (possibly v itself through a self-loop) or 0. */
static uint32_t trim2_partner(const OState *s, uint32_t v)
{
    uint32_t r = s->range[v];
    uint32_t k = 0;
    /* in-direction: the only live in-neighbour k, v -> k, and k's only
     * live in-neighbour is v */
    if (count_live_upto2(s, s->Br, s->Bc, v, r, &k) == 1) {
        for (uint32_t e = s->Fr[v]; e < s->Fr[v + 1]; e++) {
            if (s->Fc[e] == k) {
                if (count_live_upto2(s, s->Br, s->Bc, k, s->range[k], NULL) == 1) return k;
                break;
            }
        }
    }
    /* out-direction, mirrored */
    k = 0;
    if (count_live_upto2(s, s->Fr, s->Fc, v, r, &k) == 1) {
        for (uint32_t e = s->Br[v]; e < s->Br[v + 1]; e++) {
            if (s->Bc[e] == k) {
                if (count_live_upto2(s, s->Fr, s->Fc, k, s->range[k], NULL) == 1) return k;
                break;
            }
        }
    }
    return 0;
}

/* trim2 once, on the state at the start of the pass (scc_WCC.cu:792-793).
 * Both members of a pair are marked; the pair counts once, on its smaller
 * id (scc_kernels.cu:350-355). */
static void trim2_single_pass(OState *s)
{
    uint32_t n = 0;
    for (uint32_t v = 1; v <= s->V; v++) {
        if (!live(s, v)) continue;
        uint32_t k = trim2_partner(s, v);
        if (k) { s->queue[n++] = v; s->vals[v] = k; }
    }
    uint64_t pairs = 0;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t v = s->queue[i], k = s->vals[v];
        uint32_t m = v < k ? v : k;
        if (v == m) pairs++;
        s->label[v] = m;
    }
    for (uint32_t i = 0; i < n; i++) s->range[s->queue[i]] = DEADR;
    s->counts[1] += pairs;
}

/* Forward + backward reachability from the pivots already flagged in
 * fv/bv, restricted to live vertices of the same range (fwd/bwd,
 * scc_kernels.cu:360-445). */
static void fwbw_closure(OState *s, const uint32_t *seeds, uint32_t nseeds)
{
    for (int dir = 0; dir < 2; dir++) {
        const uint32_t *R = dir ? s->Br : s->Fr;
        const uint32_t *C = dir ? s->Bc : s->Fc;
        unsigned char *vis = dir ? s->bv : s->fv;
        uint32_t head = 0, tail = 0;
        for (uint32_t i = 0; i < nseeds; i++) s->queue[tail++] = seeds[i];
        while (head < tail) {
            uint32_t v = s->queue[head++];
            uint32_t r = s->range[v];
            for (uint32_t e = R[v]; e < R[v + 1]; e++) {
                uint32_t w = C[e];
                if (!vis[w] && s->range[w] == r) {
                    vis[w] = 1;
                    s->queue[tail++] = w;
                }
            }
        }
    }
}

/* Range names after a split.  The reference writes 3*range + FV + 2*BV
 * (scc_kernels.cu:138), which wraps in uint32; the restatement gives each
 * pivot three fresh names instead so that names never collide. */
static inline uint32_t split_name(uint32_t V, uint32_t p, int f, int b)
{
    return (V + 1) + 3u * p + (uint32_t)f + 2u * (uint32_t)b;
}

static int alloc_state(OState *s, uint32_t V, const uint32_t *Fr, const uint32_t *Fc,
                       const uint32_t *Br, const uint32_t *Bc)
{
    memset(s, 0, sizeof(*s));
    s->V = V; s->Fr = Fr; s->Fc = Fc; s->Br = Br; s->Bc = Bc;
    s->range = (uint32_t *)malloc((size_t)(V + 1) * 4);
    s->label = (uint32_t *)malloc((size_t)(V + 1) * 4);
    s->fv = (unsigned char *)calloc((size_t)V + 1, 1);
    s->bv = (unsigned char *)calloc((size_t)V + 1, 1);
    s->queue = (uint32_t *)malloc((size_t)(V + 1) * 4);
    s->vals = (uint32_t *)malloc((size_t)(V + 1) * 4);
    if (!s->range || !s->label || !s->fv || !s->bv || !s->queue || !s->vals) return OR_ERR_OOM;
    s->range[0] = DEADR;
    s->label[0] = 0;
    for (uint32_t v = 1; v <= V; v++) { s->range[v] = 0; s->label[v] = 0; }
    return OR_OK;
}

static void free_state(OState *s)
{
    free(s->range); free(s->label); free(s->fv); free(s->bv); free(s->queue); free(s->vals);
}

/* Relabel every vertex with the minimum id of its representative group. */
static void canonicalise(OState *s, uint32_t *labels)
{
    uint32_t V = s->V;
    uint32_t *mn = s->vals;
    for (uint32_t v = 0; v <= V; v++) mn[v] = 0xFFFFFFFFu;
    for (uint32_t v = 1; v <= V; v++) {
        uint32_t l = s->label[v];
        if (v < mn[l]) mn[l] = v;
    }
    labels[0] = 0;
    for (uint32_t v = 1; v <= V; v++) labels[v] = mn[s->label[v]];
}

/* The first FW-BW of every driver: one global pivot over live vertices
 * (pollForFirstPivot/selectFirstPivot, scc_kernels.cu:626-656), closure,
 * then update (scc_kernels.cu:124-142).  With rename=1 the non-SCC vertices
 * get split names (Hong); Slota discards ranges afterwards. */
static void first_fwbw(OState *s, int rename)
{
    uint32_t V = s->V, p = 0;
    uint64_t best = 0;
    int found = 0;
    for (uint32_t v = 1; v <= V; v++) {
        if (!live(s, v)) continue;
        uint64_t k = pivot_key(s, v);
        if (!found || k > best) { best = k; p = v; found = 1; }
    }
    if (!found) return;
    s->fv[p] = s->bv[p] = 1;
    fwbw_closure(s, &p, 1);
    s->counts[2]++;
    for (uint32_t v = 1; v <= V; v++) {
        if (!live(s, v)) continue;
        int f = s->fv[v], b = s->bv[v];
        if (f && b) { s->range[v] = DEADR; s->label[v] = p; }
        else if (rename) s->range[v] = split_name(V, p, f, b);
        else s->range[v] = 0;
        s->fv[v] = s->bv[v] = 0;
    }
}

/* "WCC" of scc_WCC.cu:830-840: every live vertex takes the minimum id over
 * the live vertices it can reach (propagateRange1 pulls the minimum over
 * out-neighbours, propagateRange2 jumps pointers; both reach this fixpoint). */
static void wcc_min_reach(OState *s)
{
    uint32_t V = s->V;
    for (uint32_t v = 1; v <= V; v++) if (live(s, v)) s->range[v] = v;
    int changed = 1;
    while (changed) {
        changed = 0;
        for (uint32_t v = V; v >= 1; v--) {
            if (!live(s, v)) continue;
            uint32_t m = s->range[v];
            for (uint32_t e = s->Fr[v]; e < s->Fr[v + 1]; e++) {
                uint32_t w = s->Fc[e];
                if (live(s, w) && s->range[w] < m) m = s->range[w];
            }
            if (m < s->range[v]) { s->range[v] = m; changed = 1; }
        }
    }
}

/* ------------------------------------------------------------------ */
/* vHong / wHong  (scc_WCC.cu:573-930; wHong :53-503 differs only in the */
/* schedule of its first FW-BW, not in what it computes)                */
/* ------------------------------------------------------------------ */

/* counts[0] = trim-1 SCCs (numberOf1Sccs), counts[1] = trim-2 pairs,
 * counts[2] = pivot SCCs; the reference prints their sum. */
int oracle_hong(uint32_t V, const uint32_t *Fr, const uint32_t *Fc,
                const uint32_t *Br, const uint32_t *Bc, int t1, int t2,
                uint32_t *labels, uint64_t counts[3])
{
    OState s;
    if (alloc_state(&s, V, Fr, Fc, Br, Bc) != OR_OK) { free_state(&s); return OR_ERR_OOM; }
    if (t1) trim1_fixpoint(&s);
    first_fwbw(&s, 1);
    if (t1) trim1_fixpoint(&s);
    if (t2) trim2_single_pass(&s);
    if (t1) trim1_fixpoint(&s);
    wcc_min_reach(&s);

    /* main loop (scc_WCC.cu:851-930): per-range pivots, FW-BW, update */
    uint64_t *best = (uint64_t *)malloc((size_t)(4ull * V + 8) * sizeof(uint64_t));
    uint32_t *seeds = (uint32_t *)malloc((size_t)(V + 1) * 4);
    if (!best || !seeds) { free(best); free(seeds); free_state(&s); return OR_ERR_OOM; }
    size_t nslots = 4ull * V + 8;
    for (;;) {
        int any = 0;
        for (uint32_t v = 1; v <= V; v++) if (live(&s, v)) { any = 1; best[s.range[v]] = 0; }
        if (!any) break;
        for (uint32_t v = 1; v <= V; v++) {
            if (!live(&s, v)) continue;
            uint64_t k = pivot_key(&s, v);
            if (k > best[s.range[v]]) best[s.range[v]] = k;
        }
        uint32_t ns = 0;
        for (uint32_t v = 1; v <= V; v++) {
            if (!live(&s, v)) continue;
            uint32_t p = 0xFFFFFFFFu - (uint32_t)(best[s.range[v]] & 0xFFFFFFFFu);
            if (p == v) { s.fv[v] = s.bv[v] = 1; seeds[ns++] = v; }
        }
        s.counts[2] += ns;
        fwbw_closure(&s, seeds, ns);
        for (uint32_t v = 1; v <= V; v++) {
            if (!live(&s, v)) continue;
            uint32_t r = s.range[v];
            uint32_t p = 0xFFFFFFFFu - (uint32_t)(best[r] & 0xFFFFFFFFu);
            int f = s.fv[v], b = s.bv[v];
            if (f && b) { s.range[v] = DEADR; s.label[v] = p; }
            else s.range[v] = split_name(V, p, f, b);
            s.fv[v] = s.bv[v] = 0;
        }
        (void)nslots;
    }
    free(best); free(seeds);
    canonicalise(&s, labels);
    memcpy(counts, s.counts, sizeof(s.counts));
    free_state(&s);
    return OR_OK;
}

/* ------------------------------------------------------------------ */
/* vSlota / wSlota  (scc_Coloring.cu:403-637 and :6-336); t2 is unused   */
/* by the reference's Slota drivers and is accepted and ignored here.   */
/* ------------------------------------------------------------------ */

int oracle_slota(uint32_t V, const uint32_t *Fr, const uint32_t *Fc,
                 const uint32_t *Br, const uint32_t *Bc, int t1, int t2,
                 uint32_t *labels, uint64_t counts[3])
{
    (void)t2;
    OState s;
    if (alloc_state(&s, V, Fr, Fc, Br, Bc) != OR_OK) { free_state(&s); return OR_ERR_OOM; }
    if (t1) trim1_single_pass(&s);
    first_fwbw(&s, 0);

    /* colouring peels (scc_Coloring.cu:590-637) */
    for (;;) {
        int any = 0;
        for (uint32_t v = 1; v <= V; v++) if (live(&s, v)) { any = 1; s.range[v] = v; }
        if (!any) break;
        /* max colour over out-neighbours to a fixpoint (colorPropagation,
         * scc_kernels.cu:539-564): colour = max id reachable */
        int changed = 1;
        while (changed) {
            changed = 0;
            for (uint32_t v = 1; v <= V; v++) {
                if (!live(&s, v)) continue;
                uint32_t m = s.range[v];
                for (uint32_t e = Fr[v]; e < Fr[v + 1]; e++) {
                    uint32_t w = Fc[e];
                    if (live(&s, w) && s.range[w] > m) m = s.range[w];
                }
                if (m > s.range[v]) { s.range[v] = m; changed = 1; }
            }
        }
        /* roots colour == id (selectPivotColoring, :567-580), then forward
         * reachability inside the colour (fwdColoring, :584-610) */
        uint32_t ns = 0;
        for (uint32_t v = 1; v <= V; v++)
            if (live(&s, v) && s.range[v] == v) { s.fv[v] = 1; s.vals[ns++] = v; }
        s.counts[2] += ns;
        uint32_t head = 0, tail = 0;
        for (uint32_t i = 0; i < ns; i++) s.queue[tail++] = s.vals[i];
        while (head < tail) {
            uint32_t v = s.queue[head++];
            uint32_t c = s.range[v];
            for (uint32_t e = Fr[v]; e < Fr[v + 1]; e++) {
                uint32_t w = Fc[e];
                if (!s.fv[w] && s.range[w] == c) { s.fv[w] = 1; s.queue[tail++] = w; }
            }
        }
        /* updateColoring (:614-623): visited vertices are done */
        for (uint32_t v = 1; v <= V; v++) {
            if (!live(&s, v)) continue;
            if (s.fv[v]) { s.label[v] = s.range[v]; s.range[v] = DEADR; }
            s.fv[v] = 0;
        }
    }
    canonicalise(&s, labels);
    memcpy(counts, s.counts, sizeof(s.counts));
    free_state(&s);
    return OR_OK;
}

/* ------------------------------------------------------------------ */
/* detectSCC (-a d): sequential restatement                           */
/* ------------------------------------------------------------------ */
/* The reference's METIS-partitioned driver (scc_WCC.cu:1000-1561) with its
 * kernels (scc_kernels.cu:21-55, 77-122, 144-185, 388-416, 447-475,
 * 665-852; identifyTransEdges and VecPushBack, scc_WCC.cu:10-50), on the
 * reference's own state: uint8 tags (scc.h:24-43) and uint32 ranges that
 * split as 3 * range + FV + 2 * BV (wrapping), with pivots kept per
 * (partition, range mod (V + 1)).  Its printed count is
 *   #trim-1 tags + #trim-2 tags + #distinct range values of every other
 *   vertex (scc_WCC.cu:1533-1546),
 * so range values that coincide count once, and the larger member of a
 * trim-2 pair (rangeSet, no tag, range 0) adds range 0 when no other vertex
 * keeps it.  Deterministic where the reference races: a pivot is the
 * largest uint32 degree product of its (partition, slot), ties to the
 * smallest id (pollForPivotsLocal's unsynchronised max); trim-2 decides on
 * the state before its pass.
 *
 * Pr: V + 2 partition ids (Pr[v] for vertex v).  counts: [trim-1, trim-2,
 * distinct ranges].  *rounds: merge rounds ("Iterations k" lines);
 * *nospace: bit r-1 set when round r printed "No space!".  Returns 0,
 * OR_ERR_OOM, or 2 when the local FW-BW loop passes V + 2 iterations (the
 * reference's loop would not end).  Fs / Bs sets are only read for the
 * ends of cross-partition edges, so they are computed for those alone. */
#define DT_FV 1u
#define DT_BV 2u
#define DT_RS 16u
#define DT_T1 32u
#define DT_T2 64u
#define DT_PIV 128u

typedef struct {
    uint32_t V;
    const uint32_t *Fr, *Fc, *Br, *Bc;
    unsigned char *tags, *aux, *occ;
    uint32_t *range, *Pr, *queue, *mark;
    uint32_t gen;
} DState;

static int d_live_same(const DState *s, const uint32_t *R, const uint32_t *C, uint32_t v)
{
    for (uint32_t e = R[v]; e < R[v + 1]; e++) {
        uint32_t w = C[e];
        if (!(s->tags[w] & DT_RS) && s->range[w] == s->range[v]) return 1;
    }
    return 0;
}

static void d_trim1(DState *s)   /* trim1 to its fixpoint (scc_kernels.cu:187-233) */
{
    for (int ch = 1; ch;) {
        ch = 0;
        for (uint32_t v = 1; v <= s->V; v++) {
            if (s->tags[v] & DT_RS) continue;
            if (!d_live_same(s, s->Br, s->Bc, v) || !d_live_same(s, s->Fr, s->Fc, v)) {
                s->tags[v] |= DT_RS | DT_T1;
                ch = 1;
            }
        }
    }
}

static uint32_t d_upto2(const DState *s, const uint32_t *R, const uint32_t *C, uint32_t x, uint32_t *first)
{
    uint32_t n = 0;
    for (uint32_t e = R[x]; e < R[x + 1]; e++) {
        uint32_t w = C[e];
        if (!(s->tags[w] & DT_RS) && s->range[w] == s->range[x]) {
            if (++n == 2) break;
            if (first) *first = w;
        }
    }
    return n;
}

static uint32_t d_trim2_partner(const DState *s, uint32_t v)   /* scc_kernels.cu:236-348 */
{
    uint32_t k = 0;
    if (d_upto2(s, s->Br, s->Bc, v, &k) == 1)
        for (uint32_t e = s->Fr[v]; e < s->Fr[v + 1]; e++)
            if (s->Fc[e] == k) {
                if (d_upto2(s, s->Br, s->Bc, k, NULL) == 1) return k;
                break;
            }
    k = 0;
    if (d_upto2(s, s->Fr, s->Fc, v, &k) == 1)
        for (uint32_t e = s->Br[v]; e < s->Br[v + 1]; e++)
            if (s->Bc[e] == k) {
                if (d_upto2(s, s->Fr, s->Fc, k, NULL) == 1) return k;
                break;
            }
    return 0;
}

/* Closure from x in direction (R, C) over vertices without rangeSet in x's
 * partition (fwdRc / bwdRc, scc_kernels.cu:806-852); marks them with a new
 * generation in s->mark and returns that generation. */
static uint32_t d_closure(DState *s, const uint32_t *R, const uint32_t *C, uint32_t x)
{
    const uint32_t gen = ++s->gen;
    uint32_t head = 0, tail = 0;
    s->mark[x] = gen;
    s->queue[tail++] = x;
    while (head < tail) {
        uint32_t u = s->queue[head++];
        for (uint32_t e = R[u]; e < R[u + 1]; e++) {
            uint32_t w = C[e];
            if (s->mark[w] != gen && !(s->tags[w] & DT_RS) && s->Pr[w] == s->Pr[u]) {
                s->mark[w] = gen;
                s->queue[tail++] = w;
            }
        }
    }
    return gen;
}

static int d_cmp_u32(const void *a, const void *b)
{
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : x > y;
}

static uint32_t d_find(uint32_t *p, uint32_t x)
{
    while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
    return x;
}

int oracle_detect(uint32_t V, const uint32_t *Fr, const uint32_t *Fc, const uint32_t *Br, const uint32_t *Bc,
                  const uint32_t *Pr_in, int t1, int t2, uint64_t *counts, uint32_t *rounds, uint32_t *nospace)
{
    const uint32_t CSize = Fr[V + 1];
    DState s;
    memset(&s, 0, sizeof(s));
    s.V = V; s.Fr = Fr; s.Fc = Fc; s.Br = Br; s.Bc = Bc;
    s.tags = (unsigned char *)calloc((size_t)V + 2, 1);
    s.aux = (unsigned char *)calloc((size_t)V + 2, 1);
    s.occ = (unsigned char *)calloc((size_t)V + 2, 1);
    s.range = (uint32_t *)calloc((size_t)V + 2, 4);
    s.Pr = (uint32_t *)malloc(((size_t)V + 2) * 4);
    s.queue = (uint32_t *)malloc(((size_t)V + 2) * 4);
    s.mark = (uint32_t *)calloc((size_t)V + 2, 4);
    uint32_t maxp = 0;
    for (uint32_t v = 1; v <= V; v++) maxp = Pr_in[v] > maxp ? Pr_in[v] : maxp;
    const size_t nslot = ((size_t)maxp + 1) * ((size_t)V + 1);
    uint32_t *best_v = (uint32_t *)malloc(nslot * 4), *best_p = (uint32_t *)malloc(nslot * 4);
    uint32_t *dsu = (uint32_t *)malloc(((size_t)V + 2) * 4), *rmax = (uint32_t *)malloc(((size_t)V + 2) * 4);
    uint32_t *Rm = (uint32_t *)malloc(((size_t)maxp + 2) * 4);
    uint32_t *tu = (uint32_t *)malloc(10001 * 4), *tv = (uint32_t *)malloc(10001 * 4);
    int rc = OR_OK;
    if (!s.tags || !s.aux || !s.occ || !s.range || !s.Pr || !s.queue || !s.mark || !best_v || !best_p || !dsu ||
        !rmax || !Rm || !tu || !tv) { rc = OR_ERR_OOM; goto out; }
    memcpy(s.Pr, Pr_in, ((size_t)V + 2) * 4);
    s.tags[0] = DT_RS;
    /* trims (scc_WCC.cu:1123-1175) */
    if (t1) d_trim1(&s);
    if (t2) {
        uint32_t n = 0;
        for (uint32_t v = 1; v <= V; v++) {
            if (s.tags[v] & DT_RS) continue;
            uint32_t k = d_trim2_partner(&s, v);
            if (k) { s.queue[n++] = v; s.mark[v] = k; }
        }
        for (uint32_t i = 0; i < n; i++) {
            uint32_t v = s.queue[i], k = s.mark[v];
            s.tags[v] |= DT_RS;
            s.tags[k] |= DT_RS;
            s.tags[v < k ? v : k] |= DT_T2;
        }
        for (uint32_t i = 0; i < n; i++) s.mark[s.queue[i]] = 0;
    }
    if (t1) d_trim1(&s);
    /* local FW-BW inside (partition, range) (scc_WCC.cu:1183-1262) */
    for (uint32_t it = 0;; it++) {
        if (it > V + 2) { rc = 2; goto out; }
        for (size_t i = 0; i < nslot; i++) { best_v[i] = 0; best_p[i] = 0; }
        for (uint32_t v = 1; v <= V; v++) {   /* pollForPivotsLocal */
            if ((s.tags[v] & DT_RS) || s.aux[v]) continue;
            size_t key = (size_t)s.Pr[v] * ((size_t)V + 1) + s.range[v] % (V + 1);
            uint32_t prod = (Fr[v + 1] - Fr[v]) * (Br[v + 1] - Br[v]);
            if (prod > best_p[key]) { best_p[key] = prod; best_v[key] = v; }
        }
        for (uint32_t v = 1; v <= V; v++) {   /* selectPivotsLocal */
            if ((s.tags[v] & DT_RS) || s.aux[v]) continue;
            size_t key = (size_t)s.Pr[v] * ((size_t)V + 1) + s.range[v] % (V + 1);
            if (best_v[key] == v) s.tags[v] = DT_FV | DT_BV | DT_PIV;
        }
        for (int dir = 0; dir < 2; dir++) {   /* fwdLocal / bwdLocal to closure */
            const uint32_t *R = dir ? Br : Fr, *C = dir ? Bc : Fc;
            const unsigned char bit = dir ? DT_BV : DT_FV;
            uint32_t head = 0, tail = 0;
            for (uint32_t v = 1; v <= V; v++)
                if (!(s.tags[v] & DT_RS) && !s.aux[v] && (s.tags[v] & bit)) s.queue[tail++] = v;
            while (head < tail) {
                uint32_t u = s.queue[head++];
                for (uint32_t e = R[u]; e < R[u + 1]; e++) {
                    uint32_t w = C[e];
                    if ((s.tags[w] & (DT_RS | bit)) || s.aux[w] || s.range[w] != s.range[u] || s.Pr[w] != s.Pr[u]) continue;
                    s.tags[w] |= bit;
                    s.queue[tail++] = w;
                }
            }
        }
        int ch = 0;   /* updateLocal */
        for (uint32_t v = 1; v <= V; v++) {
            if ((s.tags[v] & DT_RS) || s.aux[v]) continue;
            uint32_t f = (s.tags[v] & DT_FV) ? 1u : 0u, b = (s.tags[v] & DT_BV) ? 1u : 0u;
            if (f && b) s.aux[v] = 1;
            else { ch = 1; s.range[v] = 3u * s.range[v] + f + 2u * b; s.tags[v] = 0; }
        }
        if (!ch) break;
    }
    for (uint32_t v = 1; v <= V; v++)   /* resetTag over every vertex (scc_WCC.cu:1276-1333) */
        if (!(s.tags[v] & DT_RS)) s.tags[v] = 0;
    /* merge rounds (scc_WCC.cu:1347-1514) */
    *rounds = 0;
    *nospace = 0;
    for (;;) {
        uint32_t r = ++*rounds;
        for (uint32_t v = 0; v <= V; v++) s.occ[v] = 0;
        for (int dir = 0; dir < 2; dir++) {   /* computeInDegree, then computeOutDegree */
            const uint32_t *R = dir ? Fr : Br, *C = dir ? Fc : Bc;
            for (int ch = 1; ch;) {
                ch = 0;
                for (uint32_t v = 1; v <= V; v++) {
                    if ((s.tags[v] & DT_RS) || s.occ[v]) { s.occ[v] = 1; continue; }
                    uint32_t fr = (s.Pr[v] & 1u) ? s.Pr[v] - 1u : s.Pr[v] + 1u, deg = 0;
                    for (uint32_t e = R[v]; e < R[v + 1]; e++) {
                        uint32_t w = C[e];
                        if (s.occ[w] || (s.tags[w] & DT_RS)) continue;
                        if (s.Pr[w] == s.Pr[v] || s.Pr[w] == fr) deg++;
                    }
                    if (!deg) { s.occ[v] = 1; ch = 1; }
                }
            }
        }
        for (uint32_t p = 0; p <= maxp + 1; p++) Rm[p] = 0;   /* getMaxRange, shiftRange */
        for (uint32_t v = 1; v <= V; v++)
            if (!(s.tags[v] & DT_RS) && !(s.Pr[v] & 1u) && s.range[v] > Rm[s.Pr[v]]) Rm[s.Pr[v]] = s.range[v];
        for (uint32_t v = 1; v <= V; v++)
            if (!(s.tags[v] & DT_RS) && (s.Pr[v] & 1u)) s.range[v] = s.range[v] + Rm[s.Pr[v] - 1u] + 1u;
        uint32_t nt = 0, dsize = 0;   /* identifyTransEdges: at most 10001 kept (VecPushBack) */
        for (uint32_t v = 1; v <= V; v++) {
            if ((s.tags[v] & DT_RS) || s.occ[v]) continue;
            uint32_t fr = (s.Pr[v] & 1u) ? s.Pr[v] - 1u : s.Pr[v] + 1u;
            for (uint32_t e = Fr[v]; e < Fr[v + 1]; e++) {
                uint32_t w = Fc[e];
                if (!(s.tags[w] & DT_RS) && s.Pr[w] == fr && !s.occ[w]) {
                    if (dsize < 10001) { tu[nt] = v; tv[nt] = w; nt++; }
                    dsize++;
                }
            }
        }
        if (dsize >= CSize && r <= 32) *nospace |= 1u << (r - 1);
        if (dsize > 10001) nt = 0;   /* the reference's copy of dsize entries from a 10001-entry array fails */
        /* trans sets: Bs[u1_i] & Fs[u2_j] joined with Bs[u1_j] & Fs[u2_i] for every pair i < j
         * (scc_WCC.cu:1400-1433); the members of a non-empty set end with the largest range of the
         * sets they are joined through (the fixpoint of :1442-1462), i.e. the largest range of their
         * component when every set joins its members */
        for (uint32_t v = 0; v <= V; v++) dsu[v] = v;
        if (nt > 1) {
            const size_t W = ((size_t)V + 64) / 64;
            uint64_t *Fs = (uint64_t *)calloc((size_t)nt * W, 8), *Bs = (uint64_t *)calloc((size_t)nt * W, 8);
            if (!Fs || !Bs) { free(Fs); free(Bs); rc = OR_ERR_OOM; goto out; }
            for (uint32_t i = 0; i < nt; i++) {   /* Fs of the targets, Bs of the sources */
                uint32_t g = d_closure(&s, Fr, Fc, tv[i]);
                for (uint32_t v = 1; v <= V; v++) if (s.mark[v] == g) Fs[i * W + v / 64] |= 1ull << (v % 64);
                g = d_closure(&s, Br, Bc, tu[i]);
                for (uint32_t v = 1; v <= V; v++) if (s.mark[v] == g) Bs[i * W + v / 64] |= 1ull << (v % 64);
            }
            for (uint32_t i = 0; i < nt; i++)
                for (uint32_t j = i + 1; j < nt; j++) {
                    uint32_t rep = 0;
                    for (int side = 0; side < 2; side++) {
                        const uint64_t *x = Bs + (size_t)(side ? j : i) * W, *y = Fs + (size_t)(side ? i : j) * W;
                        for (size_t k = 0; k < W; k++) {
                            uint64_t m = x[k] & y[k];
                            while (m) {
                                uint32_t v = (uint32_t)(k * 64 + (uint32_t)__builtin_ctzll(m));
                                m &= m - 1;
                                if (!rep) rep = v;
                                else dsu[d_find(dsu, v)] = d_find(dsu, rep);
                            }
                        }
                    }
                }
            free(Fs);
            free(Bs);
        }
        for (uint32_t v = 1; v <= V; v++) rmax[v] = s.range[v];
        for (uint32_t v = 1; v <= V; v++) {
            uint32_t root = d_find(dsu, v);
            if (rmax[root] < s.range[v]) rmax[root] = s.range[v];
        }
        for (uint32_t v = 1; v <= V; v++) s.range[v] = rmax[d_find(dsu, v)];
        int more = 0;   /* updatePr */
        for (uint32_t v = 1; v <= V; v++) {
            if (s.tags[v] & DT_RS) continue;
            if (s.Pr[v] & 1u) { s.Pr[v] -= 1u; more = 1; }
            s.Pr[v] >>= 1;
        }
        if (!more) break;
    }
    {   /* the count (scc_WCC.cu:1533-1546) */
        uint64_t n1 = 0, n2 = 0, np = 0;
        uint32_t ns = 0;
        for (uint32_t v = 1; v <= V; v++) {
            if (s.tags[v] & DT_T1) n1++;
            else if (s.tags[v] & DT_T2) n2++;
            else s.queue[ns++] = s.range[v];
        }
        /* distinct values among the rest */
        qsort(s.queue, ns, sizeof(uint32_t), d_cmp_u32);
        for (uint32_t i = 0; i < ns; i++) np += (i == 0 || s.queue[i] != s.queue[i - 1]) ? 1u : 0u;
        counts[0] = n1; counts[1] = n2; counts[2] = np;
    }
out:
    free(s.tags); free(s.aux); free(s.occ); free(s.range); free(s.Pr); free(s.queue); free(s.mark);
    free(best_v); free(best_p); free(dsu); free(rmax); free(Rm); free(tu); free(tv);
    return rc;
}
