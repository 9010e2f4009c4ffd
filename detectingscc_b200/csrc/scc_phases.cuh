// Phases of the four SCC drivers (vHong / wHong, scc_WCC.cu:53-998; vSlota /
// wSlota, scc_Coloring.cu:6-701), rewritten as work-list passes over a
// persistent launch.  Each phase cites the reference kernel whose result it
// reproduces; the schedules differ (frontier queues instead of full-V
// sweeps, device-side convergence instead of a host round trip per level).
#pragma once
#include "scc_device.cuh"

namespace sccb {

// A vertex list: p[0..n) or, with p == nullptr, the implicit list
// base, base+1, ..., base+n-1.
struct VList {
    const uint32_t *p;
    uint32_t n;
    uint32_t base;
    __device__ __forceinline__ uint32_t at(uint32_t i) const { return p ? p[i] : base + i; }
};

// Four consecutive entries of a list for this lane (entries i0 .. i0+3): one
// 128-bit load for explicit lists (list buffers are 256-byte aligned).
__device__ __forceinline__ void load_list4(const VList &src, uint32_t i0, uint32_t (&v)[4], bool (&ok)[4])
{
    if (src.p && i0 + 3u < src.n) {
        const uint4 x = *reinterpret_cast<const uint4 *>(src.p + i0);
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
        ok[0] = ok[1] = ok[2] = ok[3] = true;
        return;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        ok[j] = i0 + (uint32_t)j < src.n;
        v[j] = ok[j] ? src.at(i0 + (uint32_t)j) : 0u;
    }
}

template <class Ex>
__device__ __forceinline__ void count_edges(Ex &ex, unsigned warp_total)
{
    if constexpr (Ex::instr) {
        if (lane_id() == 0 && warp_total) atomicAdd(&ex.ctl->t_edges, (unsigned long long)warp_total);
    }
}
template <class Ex>
__device__ __forceinline__ void count_verts(Ex &ex, bool valid)
{
    if constexpr (Ex::instr) {
        unsigned m = __ballot_sync(FULL, valid);
        if (lane_id() == 0 && m) atomicAdd(&ex.ctl->t_verts, (unsigned long long)__popc(m));
    }
}
template <class Ex>
__device__ __forceinline__ void count_verts_n(Ex &ex, unsigned n)
{
    if constexpr (Ex::instr) {
        n = __reduce_add_sync(FULL, n);
        if (lane_id() == 0 && n) atomicAdd(&ex.ctl->t_verts, (unsigned long long)n);
    }
}

// Does v have a live neighbour in range r in (R, C)?  Early exit, as in
// trim1 (scc_kernels.cu:197-222).  Self-loops count, as they do there.
template <class Ex>
__device__ __forceinline__ bool has_live(Ex &ex, const uint32_t *st, const uint32_t *__restrict__ R,
                                         const uint32_t *__restrict__ C, uint32_t v, uint32_t r, uint32_t V)
{
    uint32_t e = __ldg(&R[v]), end = __ldg(&R[v + 1]);
    bool found = false;
    uint32_t e0 = e;
    for (; e < end; e++) {
        if ((st[guard_id(__ldg(&C[e]), V, ex.ctl)] & RMASK) == r) { found = true; e++; break; }
    }
    if constexpr (Ex::instr) atomicAdd(&ex.ctl->t_edges, (unsigned long long)(e - e0));
    return found;
}

// Up to two live same-range neighbours of x in (R, C); *first gets the
// first one (scc_kernels.cu:250-261).
__device__ __forceinline__ uint32_t count_upto2(const uint32_t *st, const uint32_t *__restrict__ R,
                                                const uint32_t *__restrict__ C, uint32_t x,
                                                uint32_t r, uint32_t *first, uint32_t V, Ctl *ctl)
{
    uint32_t n = 0;
    for (uint32_t e = __ldg(&R[x]), end = __ldg(&R[x + 1]); e < end; e++) {
        uint32_t u = guard_id(__ldg(&C[e]), V, ctl);
        if ((st[u] & RMASK) == r) {
            n++;
            if (n == 2u) break;
            if (first) *first = u;
        }
    }
    return n;
}

// trim2 decision for v (scc_kernels.cu:236-348): the partner k, possibly v
// itself through a self-loop, or 0.
__device__ __forceinline__ uint32_t trim2_partner(const Graph &g, const uint32_t *st, uint32_t v, uint32_t r, Ctl *c)
{
    uint32_t k = 0;
    if (count_upto2(st, g.Br, g.Bc, v, r, &k, g.V, c) == 1u) {
        for (uint32_t e = __ldg(&g.Fr[v]), end = __ldg(&g.Fr[v + 1]); e < end; e++) {
            if (__ldg(&g.Fc[e]) == k) {
                if (count_upto2(st, g.Br, g.Bc, k, r, nullptr, g.V, c) == 1u) return k;
                break;
            }
        }
    }
    k = 0;
    if (count_upto2(st, g.Fr, g.Fc, v, r, &k, g.V, c) == 1u) {
        for (uint32_t e = __ldg(&g.Br[v]), end = __ldg(&g.Br[v + 1]); e < end; e++) {
            if (__ldg(&g.Bc[e]) == k) {
                if (count_upto2(st, g.Fr, g.Fc, k, r, nullptr, g.V, c) == 1u) return k;
                break;
            }
        }
    }
    return 0;
}

// ---------------------------------------------------------------------
// init: every vertex live in range 0 (the reference's cudaMemset of range
// and tags, scc_WCC.cu:630-631); optionally fold the first-pivot key.
// ---------------------------------------------------------------------
template <class Ex>
__device__ bool ph_init(Ex &ex, const Graph &g, const Work &w, bool fold_pivot)
{
    // Also checks the offsets (the reference layout: Fr[0] = Fr[1] = 0,
    // non-decreasing, Fr[V+1] = E, load.cpp:55-77; same for Br).  A bad
    // graph sets the error before the barrier, so no later pass runs.
    // Four ids per lane: 128-bit offset loads and state stores.
    return run_pass(ex, PH_INIT, [&](unsigned, unsigned) {
        unsigned long long best = 0;
        if (ex.leader() && (g.Fr[0] != 0u || g.Fr[1] != 0u || g.Br[0] != 0u || g.Br[1] != 0u ||
                            g.Fr[g.V + 1] != g.E || g.Br[g.V + 1] != g.E))
            set_error(ex.ctl, E_BAD_GRAPH, 62);
        bool bad = false;
        uint32_t dmax = 0;
        for (uint32_t i0 = ex.tid() * 4u; i0 <= g.V; i0 += ex.nthr() * 4u) {
            uint32_t f[5], b[5];
            load_off5(g.Fr, i0, g.V, g.vec, f);
            load_off5(g.Br, i0, g.V, g.vec, b);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint32_t i = i0 + (uint32_t)j;
                if (i <= g.V) {
                    bad |= f[j] > f[j + 1] || b[j] > b[j + 1];
                    dmax = max(dmax, max(f[j + 1] - f[j], b[j + 1] - b[j]));
                    if (fold_pivot && i != 0u) {
                        unsigned long long k = ((unsigned long long)((f[j + 1] - f[j]) * (b[j + 1] - b[j])) << 32) |
                                               (0xFFFFFFFFu - i);
                        best = k > best ? k : best;
                    }
                }
            }
            if (i0 + 3u <= g.V) {
                *reinterpret_cast<uint4 *>(w.st + i0) = make_uint4(i0 == 0u ? DEAD : 0u, 0u, 0u, 0u);
                *reinterpret_cast<uint4 *>(w.stamp + i0) = make_uint4(0u, 0u, 0u, 0u);
            } else {
                for (uint32_t i = i0; i <= g.V; i++) {
                    w.st[i] = (i == 0u) ? DEAD : 0u;
                    w.stamp[i] = 0u;
                }
            }
        }
        if (bad) set_error(ex.ctl, E_BAD_GRAPH, 61);
        if (fold_pivot) block_max_atomic(best, &w.pivkey[0], dmax, Ex::nbq > 2 ? &ex.ctl->maxdeg : nullptr);
        else if constexpr (Ex::nbq > 2) block_max_atomic32(dmax, &ex.ctl->maxdeg);
    });
}

// ---------------------------------------------------------------------
// init and trim1-once in one sweep (vSlota / wSlota with trim1): with every
// vertex live in range 0, trim1 is decided by the degrees alone, so the
// offsets the init pass validates also decide each vertex's first state.
// Four ids per lane: 128-bit offset loads and 128-bit stores of st and
// label (a trimmed vertex is labelled with itself, LBL_SELF).  Stamps are
// cleared later for the few vertices that need them (ph_slota_first_update)
// and smin entries when their representative is seeded, so this sweep
// writes two vertex arrays, not four.  Survivors are compacted into Lout and
// bid for the first pivot.  A bad graph sets the error before the barrier,
// as in ph_init.
// ---------------------------------------------------------------------
template <class Ex>
__device__ bool ph_init_trim1(Ex &ex, const Graph &g, const Work &w, uint32_t *Lout)
{
    return run_pass(ex, PH_TRIM1_ONCE, [&](unsigned, unsigned nxt) {
        if (ex.leader() && (g.Fr[0] != 0u || g.Fr[1] != 0u || g.Br[0] != 0u || g.Br[1] != 0u ||
                            g.Fr[g.V + 1] != g.E || g.Br[g.V + 1] != g.E))
            set_error(ex.ctl, E_BAD_GRAPH, 62);
        unsigned long long best = 0;
        unsigned ntrim = 0;
        bool bad = false;
        uint32_t dmax = 0;
        for (uint32_t base = ex.wid() * 128u; base <= g.V; base += ex.nwarps() * 128u) {
            const uint32_t i0 = base + 4u * lane_id();
            uint32_t f[5], b[5];
            if (i0 <= g.V) {
                load_off5(g.Fr, i0, g.V, g.vec, f);
                load_off5(g.Br, i0, g.V, g.vec, b);
            } else {
#pragma unroll
                for (int j = 0; j < 5; j++) f[j] = b[j] = 0u;
            }
            uint32_t st4[4], lb4[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint32_t v = i0 + (uint32_t)j;
                const bool valid = v >= 1u && v <= g.V;
                bool surv = false;
                st4[j] = DEAD;
                lb4[j] = v;
                if (v <= g.V) bad |= f[j] > f[j + 1] || b[j] > b[j + 1];
                if (valid) {
                    const uint32_t indeg = b[j + 1] - b[j], outdeg = f[j + 1] - f[j];
                    dmax = max(dmax, max(indeg, outdeg));
                    if (indeg == 0u || outdeg == 0u) {
                        lb4[j] = v | LBL_SELF;   // a trimmed vertex is its own SCC
                        ntrim++;
                    } else {
                        surv = true;
                        st4[j] = 0u;
                        unsigned long long k = ((unsigned long long)(outdeg * indeg) << 32) | (0xFFFFFFFFu - v);
                        best = k > best ? k : best;
                    }
                }
                bq_push(0, surv, v, w.qcap, Lout, &ex.lc(nxt)[C_LIST], g.V, ex.ctl, 10);
            }
            if (i0 + 3u <= g.V) {
                *reinterpret_cast<uint4 *>(w.st + i0) = make_uint4(st4[0], st4[1], st4[2], st4[3]);
                *reinterpret_cast<uint4 *>(w.label + i0) = make_uint4(lb4[0], lb4[1], lb4[2], lb4[3]);
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const uint32_t i = i0 + (uint32_t)j;
                    if (i <= g.V) {
                        w.st[i] = st4[j];
                        w.label[i] = lb4[j];
                    }
                }
            }
            count_verts_n(ex, i0 <= g.V ? min(4u, g.V + 1u - i0) : 0u);
        }
        if (bad) set_error(ex.ctl, E_BAD_GRAPH, 61);
        ntrim = __reduce_add_sync(FULL, ntrim);
        if (lane_id() == 0 && ntrim) atomicAdd(&ex.ctl->n_trim1, (unsigned long long)ntrim);
        block_max_atomic(best, &w.pivkey[0], dmax, Ex::nbq > 2 ? &ex.ctl->maxdeg : nullptr);
        bq_flush(1, w.qcap, Lout, &ex.lc(nxt)[C_LIST], nullptr, nullptr, g.V, ex.ctl);
    });
}

// ---------------------------------------------------------------------
// trim1 iterated to its fixpoint (vHong / wHong, scc_WCC.cu:680-687,
// :773-780, :808-815).  Pass 0 checks src0; a trimmed vertex queues its
// live same-range neighbours for the next pass (stamp-deduplicated), so
// later passes only recheck vertices that lost a neighbour.
// ---------------------------------------------------------------------
template <class Ex>
__device__ bool ph_trim1_fix(Ex &ex, const Graph &g, const Work &w, VList src0, bool all_live)
{
    uint32_t nq = 0;
    bool first = true;
    for (unsigned it = 0;; it++) {
        if (it > g.V + 2u) { if (ex.leader()) set_error(ex.ctl, E_NOT_CONVERGED, 30); return false; }
        bool ok = run_pass(ex, PH_TRIM1_FIX, [&](unsigned, unsigned nxt) {
            const unsigned par = ex.gl & 1u;
            const uint32_t tag = ex.gl + 1u;
            VList src = first ? src0 : VList{w.Q[0][par ^ 1u], nq, 0u};
            for (uint32_t base = ex.wid() * 32u; base < src.n; base += ex.nwarps() * 32u) {
                uint32_t i = base + lane_id();
                bool valid = i < src.n, trim = false;
                uint32_t v = valid ? src.at(i) : 0u, r = 0u;
                if (valid) {
                    uint32_t s = w.st[v];
                    if (s != DEAD) {
                        r = s & RMASK;
                        if (first && all_live)   // every vertex live in range 0: degrees decide
                            trim = __ldg(&g.Br[v + 1]) == __ldg(&g.Br[v]) || __ldg(&g.Fr[v + 1]) == __ldg(&g.Fr[v]);
                        else
                            trim = !has_live(ex, w.st, g.Br, g.Bc, v, r, g.V) ||
                                   !has_live(ex, w.st, g.Fr, g.Fc, v, r, g.V);
                        if (trim) { w.st[v] = DEAD; w.label[v] = v | LBL_SELF; }
                    }
                }
                count_verts(ex, valid);
                unsigned m = __ballot_sync(FULL, trim);
                if (lane_id() == 0 && m) atomicAdd(&ex.ctl->n_trim1, (unsigned long long)__popc(m));
                if (m == 0u) continue;
                // queue the live same-range neighbours of the trimmed vertices
                // (they lost an in- or out-neighbour): the warp walks all their
                // lists together, 64 entries per step
                auto fn2 = [&](bool v0, uint32_t u0, uint32_t r0, bool v1, uint32_t u1, uint32_t r1) {
                    if (v0) u0 = guard_id(u0, g.V, ex.ctl);
                    if (v1) u1 = guard_id(u1, g.V, ex.ctl);
                    const bool p0 = v0 && (w.st[u0] & RMASK) == r0 && stamp_claim(w.stamp, u0, tag);
                    const bool p1 = v1 && (w.st[u1] & RMASK) == r1 && stamp_claim(w.stamp, u1, tag);
                    bq_push(0, p0, u0, w.qcap, w.Q[0][par], &ex.lc(nxt)[C_FQ], g.V, ex.ctl, 11);
                    bq_push(0, p1, u1, w.qcap, w.Q[0][par], &ex.lc(nxt)[C_FQ], g.V, ex.ctl, 11);
                };
#pragma unroll
                for (int dir = 0; dir < 2; dir++) {
                    const uint32_t *R = dir ? g.Br : g.Fr;
                    const uint32_t *C = dir ? g.Bc : g.Fc;
                    const uint32_t beg = trim ? __ldg(&R[v]) : 0u;
                    const uint32_t deg = trim ? __ldg(&R[v + 1]) - beg : 0u;
                    count_edges(ex, lbs_expand2(beg, deg, r, C, fn2));
                }
            }
            bq_flush(1, w.qcap, w.Q[0][par], &ex.lc(nxt)[C_FQ], nullptr, nullptr, g.V, ex.ctl);
        });
        if (!ok) return false;
        first = false;
        nq = last_count(ex, C_FQ);
        if (nq == 0u) return true;
    }
}

// ---------------------------------------------------------------------
// trim2 once, decided on the state before the pass (scc_WCC.cu:792-793,
// scc_kernels.cu:236-357).  Both members are marked; the pair counts once,
// on its smaller id.  The reference marks both members with unsynchronised
// byte writes (scc_kernels.cu:350-354) and can lose the trim2 tag.
// ---------------------------------------------------------------------
template <class Ex>
__device__ bool ph_trim2(Ex &ex, const Graph &g, const Work &w, VList src)
{
    bool ok = run_pass(ex, PH_TRIM2, [&](unsigned, unsigned nxt) {
        const unsigned par = ex.gl & 1u;
        for (uint32_t base = ex.wid() * 32u; base < src.n; base += ex.nwarps() * 32u) {
            uint32_t i = base + lane_id();
            bool valid = i < src.n, hit = false, cnt = false;
            uint32_t v = valid ? src.at(i) : 0u;
            if (valid) {
                uint32_t s = w.st[v];
                if (s != DEAD) {
                    uint32_t k = trim2_partner(g, w.st, v, s & RMASK, ex.ctl);
                    if (k) {
                        hit = true;
                        cnt = v <= k;
                        w.label[v] = (v < k ? v : k) | LBL_SELF;
                    }
                }
            }
            count_verts(ex, valid);
            unsigned m = __ballot_sync(FULL, cnt);
            if (lane_id() == 0 && m) atomicAdd(&ex.ctl->n_trim2, (unsigned long long)__popc(m));
            bq_push(0, hit, v, w.qcap, w.Q[0][par], &ex.lc(nxt)[C_LIST], g.V, ex.ctl, 12);
        }
        bq_flush(1, w.qcap, w.Q[0][par], &ex.lc(nxt)[C_LIST], nullptr, nullptr, g.V, ex.ctl);
    });
    if (!ok) return false;
    const uint32_t nT = last_count(ex, C_LIST);
    return run_pass(ex, PH_TRIM2_APPLY, [&](unsigned, unsigned) {
        const uint32_t *T = w.Q[0][(ex.gl & 1u) ^ 1u];
        for (uint32_t i = ex.tid(); i < nT; i += ex.nthr()) w.st[T[i]] = DEAD;
    });
}

// ---------------------------------------------------------------------
// Frontier expansion of one direction for the lanes of a warp.  A lane with
// act holds vertex v of range r; its neighbours that are live, in range r
// and not yet visited in this direction are claimed with atomicOr and
// appended to the next frontier (warp ballot compaction).  Vertices with
// more than HEAVY_T entries are cut into CH-entry chunks for the next pass.
// This is fwd/bwd (scc_kernels.cu:360-445) and fwd_warp/bwd_warp
// (include/scc_kernels.h:46-105) over a queue instead of a full sweep.
// ---------------------------------------------------------------------
template <class Ex>
__device__ __forceinline__ void bfs_edge_visit(Ex &ex, const Graph &g, const Work &w, int dir, bool valid,
                                               uint32_t nbr, uint32_t r, unsigned par, unsigned nxt, bool cnt)
{
    const uint32_t bit = dir ? BVB : FVB;
    bool claim = false;
    uint32_t done = 0xFFFFFFFFu;
    if (valid) {
        nbr = guard_id(nbr, g.V, ex.ctl);
        uint32_t s = w.st[nbr];
        if ((s & (RMASK | bit)) == r) {
            const uint32_t o = atomicOr(&w.st[nbr], bit);
            claim = !(o & bit);
            done = completed(o, bit, nbr);
        }
    }
    fold_completed(done);
    const uint32_t *Rn = dir ? g.Br : g.Fr;
    if (cnt) bq_add_edges((unsigned)dir, claim ? __ldg(&Rn[nbr + 1]) - __ldg(&Rn[nbr]) : 0u);
    bq_push((unsigned)dir, claim, nbr, w.qcap, w.Q[dir][par], &ex.lc(nxt)[C_FQ + dir], g.V, ex.ctl, 13);
}

// Two adjacency entries per lane: both gathers and both claims are issued
// before either append, so every lane keeps two requests in flight.  cnt
// (uniform over the CTA) adds the claimed vertices' degrees to the pass's
// frontier-edge tally; a pass whose claims cannot reach the bottom-up
// threshold skips those offset gathers.
template <class Ex>
__device__ __forceinline__ void bfs_edge_visit2(Ex &ex, const Graph &g, const Work &w, int dir, bool v0, uint32_t n0,
                                                uint32_t r0, bool v1, uint32_t n1, uint32_t r1, unsigned par,
                                                unsigned nxt, bool cnt)
{
    const uint32_t bit = dir ? BVB : FVB;
    if (v0) n0 = guard_id(n0, g.V, ex.ctl);
    if (v1) n1 = guard_id(n1, g.V, ex.ctl);
    const uint32_t s0 = v0 ? w.st[n0] : DEAD;
    const uint32_t s1 = v1 ? w.st[n1] : DEAD;
    const bool t0 = v0 && (s0 & (RMASK | bit)) == r0;
    const bool t1 = v1 && (s1 & (RMASK | bit)) == r1;
    const uint32_t o0 = t0 ? atomicOr(&w.st[n0], bit) : bit;
    const uint32_t o1 = t1 ? atomicOr(&w.st[n1], bit) : bit;
    const bool c0 = !(o0 & bit), c1 = !(o1 & bit);
    fold_completed(min(c0 ? completed(o0, bit, n0) : 0xFFFFFFFFu, c1 ? completed(o1, bit, n1) : 0xFFFFFFFFu));
    // edges the claimed vertices will expand next (direction-switch rule)
    if (cnt) {
        const uint32_t *Rn = dir ? g.Br : g.Fr;
        unsigned e = 0;
        if (c0) e += __ldg(&Rn[n0 + 1]) - __ldg(&Rn[n0]);
        if (c1) e += __ldg(&Rn[n1 + 1]) - __ldg(&Rn[n1]);
        bq_add_edges((unsigned)dir, e);
    }
    bq_push((unsigned)dir, c0, n0, w.qcap, w.Q[dir][par], &ex.lc(nxt)[C_FQ + dir], g.V, ex.ctl, 13);
    bq_push((unsigned)dir, c1, n1, w.qcap, w.Q[dir][par], &ex.lc(nxt)[C_FQ + dir], g.V, ex.ctl, 13);
}

template <class Ex>
__device__ __forceinline__ void bfs_expand_lanes(Ex &ex, const Graph &g, const Work &w, int dir, uint32_t v,
                                                 bool act, uint32_t r, int lw, unsigned par, unsigned nxt,
                                                 bool cnt = true)
{
    const uint32_t *R = dir ? g.Br : g.Fr;
    const uint32_t *C = dir ? g.Bc : g.Fc;
    uint32_t beg = 0, deg = 0;
    if (act) { beg = __ldg(&R[v]); deg = __ldg(&R[v + 1]) - beg; }
    bool heavy = deg > HEAVY_T;
    uint32_t nch = heavy ? (deg + CH - 1u) / CH : 0u;
    if (lw > 0 && (lane_id() & ((1u << lw) - 1u)) != 0u) nch = 0u;
    warp_push_chunks(v, nch, w.H[dir][par], &ex.lc(nxt)[C_FH + dir], w.hcap, ex.ctl);
    if (heavy) deg = 0u;
    unsigned tot;
    if (lw < 0) {
        auto fn2 = [&](bool v0, uint32_t n0, uint32_t r0, bool v1, uint32_t n1, uint32_t r1) {
            bfs_edge_visit2(ex, g, w, dir, v0, n0, r0, v1, n1, r1, par, nxt, cnt);
        };
        tot = lbs_expand2(beg, deg, r, C, fn2);
    } else {
        auto fn = [&](bool valid, uint32_t nbr, uint32_t rr) {
            bfs_edge_visit(ex, g, w, dir, valid, nbr, rr, par, nxt, cnt);
        };
        tot = vw_expand(beg, deg, r, (unsigned)lw, C, fn);
    }
    count_edges(ex, tot);
}

// Top-down expansion with the virtual-warp schedule (W = 1 << lw lanes per
// vertex, the reference's fwd_warp/bwd_warp), VWK frontier vertices per
// lane group in the same steps.
constexpr int VWK = 4;
template <class Ex>
__device__ __forceinline__ void bfs_expand_vwk(Ex &ex, const Graph &g, const Work &w, int dir,
                                               const uint32_t (&v)[VWK], const bool (&act)[VWK],
                                               const uint32_t (&r)[VWK], int lw, unsigned par, unsigned nxt,
                                               bool cnt)
{
    const uint32_t *R = dir ? g.Br : g.Fr;
    const uint32_t *C = dir ? g.Bc : g.Fc;
    const bool lead = (lane_id() & ((1u << lw) - 1u)) == 0u;
    uint32_t beg[VWK], deg[VWK];
#pragma unroll
    for (int j = 0; j < VWK; j++) {
        beg[j] = act[j] ? __ldg(&R[v[j]]) : 0u;
        deg[j] = act[j] ? __ldg(&R[v[j] + 1]) - beg[j] : 0u;
    }
#pragma unroll
    for (int j = 0; j < VWK; j++) {
        const bool heavy = deg[j] > HEAVY_T;
        warp_push_chunks(v[j], heavy && lead ? (deg[j] + CH - 1u) / CH : 0u, w.H[dir][par],
                         &ex.lc(nxt)[C_FH + dir], w.hcap, ex.ctl);
        if (heavy) deg[j] = 0u;
    }
    auto fn = [&](int j, bool v0, uint32_t n0, bool v1, uint32_t n1) {
        bfs_edge_visit2(ex, g, w, dir, v0, n0, r[j], v1, n1, r[j + 1], par, nxt, cnt);
    };
    count_edges(ex, vw_expandK<VWK>(beg, deg, (unsigned)lw, C, fn));
}

// One CH-entry chunk of a heavy vertex, expanded by the whole warp.
template <class Ex, class Fn>
__device__ __forceinline__ void chunk_expand(Ex &ex, const uint32_t *__restrict__ R, const uint32_t *__restrict__ C,
                                             uint2 hc, uint32_t aux, Fn &&fn)
{
    uint32_t beg = __ldg(&R[hc.x]) + hc.y * CH;
    uint32_t end = min(__ldg(&R[hc.x + 1]), beg + CH);
    for (uint32_t k = lane_id(); k < CH; k += 64u) {
        const uint32_t e0 = beg + k, e1 = e0 + 32u;
        const bool v0 = e0 < end, v1 = e1 < end;
        const uint32_t n0 = v0 ? __ldg(&C[e0]) : 0u;
        const uint32_t n1 = v1 ? __ldg(&C[e1]) : 0u;
        fn(v0, n0, aux, v1, n1, aux);
    }
    count_edges(ex, end > beg ? end - beg : 0u);
}

// Bottom-up step over 64 vertices, both directions at once: entries
// k*64 .. k*64+63 of `src` (the scope list, or the id range 1..V when the
// scope holds most live vertices: coalesced state and offset loads, no list
// indirection), two per lane.  Every lane keeps up to four searches in
// flight (2 vertices x forward/backward), each testing two adjacency
// entries per step, so a lane waits on one round of gathers for all of
// them; a list longer than 32 entries gets its first 8 entries tested by
// the lane (a visited neighbour is usually among the first, lowest ids) and
// the rest by the whole warp.  A live vertex outside the scope can only
// find a visited neighbour of its own range if its range is being
// searched, so walking ids reaches the same set as walking the scope.
//
// With sout set (whole-GPU policy), every live vertex of the item that is
// still unvisited in a direction of the search is appended to sout (staging
// queue 2): the scope of the next bottom-up step, which then walks only
// those instead of the whole scope.
template <class Ex>
__device__ __forceinline__ void bfs_pull2(Ex &ex, const Graph &g, const Work &w, bool puf, bool pub, bool bw,
                                          VList src, uint32_t k, unsigned par, unsigned nxt, uint32_t *sout)
{
    constexpr uint32_t MF = RMASK | FVB, MB = RMASK | BVB;
    uint32_t v[2], s[2], pos[4], end[4], want[4];
    bool on[4], found[4], ok[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const uint32_t i = k * 64u + 32u * (uint32_t)h + lane_id();
        ok[h] = i < src.n;
        v[h] = ok[h] ? src.at(i) : 0u;
    }
#pragma unroll
    for (int h = 0; h < 2; h++) s[h] = ok[h] ? w.st[v[h]] : DEAD;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const bool live = s[h] != DEAD;
        const bool nf = puf && live && !(s[h] & FVB);   // forward: a visited in-neighbour
        const bool nb = pub && live && !(s[h] & BVB);   // backward: a visited out-neighbour
        pos[2 * h] = nf ? __ldg(&g.Br[v[h]]) : 0u;
        end[2 * h] = nf ? __ldg(&g.Br[v[h] + 1u]) : 0u;
        pos[2 * h + 1] = nb ? __ldg(&g.Fr[v[h]]) : 0u;
        end[2 * h + 1] = nb ? __ldg(&g.Fr[v[h] + 1u]) : 0u;
        want[2 * h] = (s[h] & RMASK) | FVB;
        want[2 * h + 1] = (s[h] & RMASK) | BVB;
    }
    unsigned scanned = 0;
    uint32_t lim[4];   // the lane scans a list to its end if it is short, else its first entries
    const uint32_t first = min(8u, w.pull_lane);
#pragma unroll
    for (int t = 0; t < 4; t++) {
        found[t] = false;
        on[t] = end[t] > pos[t];
        lim[t] = end[t] - pos[t] <= w.pull_lane ? end[t] : pos[t] + first;
    }
    // by the lane: two entries of every open search per step (a visited
    // neighbour is usually among the first entries, the lowest ids)
    while (on[0] || on[1] || on[2] || on[3]) {
        uint32_t c0[4], c1[4];
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const uint32_t *C = (t & 1) ? g.Fc : g.Bc;
            c0[t] = on[t] ? __ldg(&C[pos[t]]) : 0u;
            c1[t] = on[t] && pos[t] + 1u < end[t] ? __ldg(&C[pos[t] + 1u]) : 0u;
        }
#pragma unroll
        for (int t = 0; t < 4; t++) {
            if (!on[t]) continue;
            const uint32_t m = (t & 1) ? MB : MF;
            const uint32_t a = w.st[guard_id(c0[t], g.V, ex.ctl)];
            const uint32_t b = pos[t] + 1u < end[t] ? w.st[guard_id(c1[t], g.V, ex.ctl)] : DEAD;
            if constexpr (Ex::instr) scanned += pos[t] + 1u < end[t] ? 2u : 1u;
            if ((a & m) == want[t] || (b & m) == want[t]) {
                found[t] = true;
                on[t] = false;
            } else {
                pos[t] += 2u;
                on[t] = pos[t] < lim[t];
            }
        }
    }
    // the rest of long lists by the whole warp, one search at a time
#pragma unroll
    for (int t = 0; t < 4; t++) {
        unsigned hm = __ballot_sync(FULL, !found[t] && end[t] > pos[t]);
        const uint32_t *C = (t & 1) ? g.Fc : g.Bc;
        const uint32_t m = (t & 1) ? MB : MF;
        while (hm) {
            const unsigned j = __ffs(hm) - 1u;
            hm &= hm - 1u;
            const uint32_t bj = __shfl_sync(FULL, pos[t], j), ej = __shfl_sync(FULL, end[t], j);
            const uint32_t wj = __shfl_sync(FULL, want[t], j);
            for (uint32_t b = bj; b < ej; b += 32u) {
                const uint32_t e = b + lane_id();
                const bool hit = e < ej && (w.st[guard_id(__ldg(&C[e]), g.V, ex.ctl)] & m) == wj;
                if constexpr (Ex::instr) scanned += lane_id() == 0 ? min(32u, ej - b) : 0u;
                if (__ballot_sync(FULL, hit)) {
                    if (lane_id() == j) found[t] = true;
                    break;
                }
            }
        }
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const uint32_t bits = (found[2 * h] ? FVB : 0u) | (found[2 * h + 1] ? BVB : 0u);
        fold_completed(bits ? completed(atomicOr(&w.st[v[h]], bits), bits, v[h]) : 0xFFFFFFFFu);
        // frontier edges of the next level: out-degree forward, in-degree backward
        if (puf) bq_add_edges(0u, found[2 * h] ? __ldg(&g.Fr[v[h] + 1u]) - __ldg(&g.Fr[v[h]]) : 0u);
        if (pub) bq_add_edges(1u, found[2 * h + 1] ? __ldg(&g.Br[v[h] + 1u]) - __ldg(&g.Br[v[h]]) : 0u);
        count_verts(ex, ok[h]);
        if (puf) bq_push(0u, found[2 * h], v[h], w.qcap, w.Q[0][par], &ex.lc(nxt)[C_FQ], g.V, ex.ctl, 19);
        if (pub) bq_push(1u, found[2 * h + 1], v[h], w.qcap, w.Q[1][par], &ex.lc(nxt)[C_BQ], g.V, ex.ctl, 19);
        if (Ex::nbq > 2 && sout) {
            const bool fv = (s[h] & FVB) || found[2 * h], bv = (s[h] & BVB) || found[2 * h + 1];
            const bool keep = s[h] != DEAD && !(fv && (bv || !bw));
            bq_push(2u, keep, v[h], w.qcap, sout, &ex.lc(nxt)[C_SCOPE], g.V, ex.ctl, 25);
        }
    }
    if constexpr (Ex::instr) {
        unsigned t = __reduce_add_sync(FULL, scanned);
        count_edges(ex, t);
    }
}

// Seed predicates for the first BFS pass.
// A seed takes list entry x: operator() says whether it seeds, vert() which
// vertex it seeds.
struct SeedOne {      // the single first pivot
    uint32_t p;
    __device__ __forceinline__ bool operator()(const Work &, uint32_t v) const { return v == p; }
    __device__ __forceinline__ uint32_t vert(const Work &, uint32_t x) const { return x; }
};
struct SeedRoot {     // colouring roots (selectPivotColoring, scc_kernels.cu:567-580)
    __device__ __forceinline__ bool operator()(const Work &w, uint32_t v) const { return w.st[v] == v; }
    __device__ __forceinline__ uint32_t vert(const Work &, uint32_t x) const { return x; }
};
struct SeedRanges {   // per-range pivots (selectPivots, scc_kernels.cu:4-19), walked over the
                      // list of live ranges instead of every live vertex
    __device__ __forceinline__ bool operator()(const Work &w, uint32_t r) const { return w.pivkey[r] != 0ull; }
    __device__ __forceinline__ uint32_t vert(const Work &w, uint32_t r) const { return key_vertex(w.pivkey[r]); }
};

// Forward (and backward) reachability to closure.  Pass 0 walks src, tests
// the seed predicate, flags seeds and expands them.  Each later pass picks,
// per direction, top-down (expand the frontier queue and the heavy chunks)
// or bottom-up over `scope` (the vertices the search can reach) when the
// frontier's vertices have more than bu_k * scope.n edges to expand.  lw < 0 selects the
// load-balanced warp schedule for top-down steps, lw >= 0 the virtual-warp
// schedule with W = 1 << lw.
//
// On the whole-GPU policy every bottom-up step also lists the vertices of
// its scope still unvisited in some direction (into w.S[0], w.S[1] in
// turn): the next bottom-up step walks that shorter list, and the Beamer
// rule weighs the frontier against it.  *last (optional) receives the scope
// at the end: every live vertex of the original scope that is not visited
// in both directions is in it.
template <class Ex, class Seed>
__device__ bool ph_bfs(Ex &ex, const Graph &g, const Work &w, VList src, Seed seed, bool bw, int lw, VList scope,
                       VList *last = nullptr)
{
    unsigned nshrink = 0;
    const unsigned gsz = (lw < 0) ? 32u : (32u >> lw);
    const bool single = src.n == 1u && src.p == nullptr;
    bool ok = run_pass(ex, PH_BFS0, [&](unsigned, unsigned nxt) {
        const unsigned par = ex.gl & 1u;
        const unsigned ng = single ? 0u : (src.n + gsz - 1u) / gsz;
        const uint32_t bits = bw ? (FVB | BVB) : FVB;
        if (single && seed(w, src.base)) {
            // one seed (the first pivot, usually the largest hub): every warp
            // takes CH-entry chunks of its out- and in-list in this pass
            const uint32_t p = src.base;
            if (ex.leader()) {
                if (completed(atomicOr(&w.st[p], bits), bits, p) == p) atomicMin(cta_first_min(), p);
                atomicAdd(&ex.ctl->n_pivot, 1ull);
                w.smin[p] = p;   // p represents its SCC: the update passes fold the members in
            }
            // 64-entry pieces, one per warp, so the hub's lists spread over
            // the whole grid in one round of gathers
            const uint32_t r = w.st[p] & RMASK;
            const uint32_t fb = __ldg(&g.Fr[p]), fe = __ldg(&g.Fr[p + 1]);
            const uint32_t bb = bw ? __ldg(&g.Br[p]) : 0u, be = bw ? __ldg(&g.Br[p + 1]) : 0u;
            const uint32_t nfc = (fe - fb + 63u) / 64u, nbc = (be - bb + 63u) / 64u;
            for (uint32_t c = ex.wid(); c < nfc + nbc; c += ex.nwarps()) {
                const int dir = c < nfc ? 0 : 1;
                const uint32_t beg = dir ? bb + (c - nfc) * 64u : fb + c * 64u;
                const uint32_t end = min(beg + 64u, dir ? be : fe);
                const uint32_t *C = dir ? g.Bc : g.Fc;
                const uint32_t e0 = beg + lane_id(), e1 = e0 + 32u;
                const bool v0 = e0 < end, v1 = e1 < end;
                const uint32_t n0 = v0 ? __ldg(&C[e0]) : 0u, n1 = v1 ? __ldg(&C[e1]) : 0u;
                bfs_edge_visit2(ex, g, w, dir, v0, n0, r, v1, n1, r, par, nxt, true);
                count_edges(ex, end - beg);
            }
        }
        for (uint32_t it = ex.wid(); it < ng; it += ex.nwarps()) {
            unsigned slot = (lw < 0) ? lane_id() : (lane_id() >> lw);
            uint32_t i = it * gsz + slot;
            bool valid = i < src.n;
            const uint32_t x = valid ? src.at(i) : 0u;
            bool act = valid && seed(w, x);
            uint32_t v = act ? seed.vert(w, x) : x;
            bool lead = (lw <= 0) || ((lane_id() & ((1u << lw) - 1u)) == 0u);
            uint32_t r = 0;
            uint32_t done = 0xFFFFFFFFu;
            if (act && lead) {
                const uint32_t o = atomicOr(&w.st[v], bits);
                done = completed(o, bits, v);
                r = o & RMASK;
                w.smin[v] = v;   // v represents its SCC from here on
            }
            fold_completed(done);
            if (lw > 0) r = __shfl_sync(FULL, r, lane_id() & ~((1u << lw) - 1u));
            unsigned m = __ballot_sync(FULL, act && lead);
            if (lane_id() == 0 && m) atomicAdd(&ex.ctl->n_pivot, (unsigned long long)__popc(m));
            count_verts(ex, valid && lead);
            bfs_expand_lanes(ex, g, w, 0, v, act, r, lw, par, nxt);
            if (bw) bfs_expand_lanes(ex, g, w, 1, v, act, r, lw, par, nxt);
        }
        bq_flush(2, w.qcap, w.Q[0][par], &ex.lc(nxt)[C_FQ], w.Q[1][par], &ex.lc(nxt)[C_BQ], g.V, ex.ctl,
                 &ex.lc(nxt)[C_FE], &ex.lc(nxt)[C_BE]);
    });
    if (!ok) return false;
    // The claims of a pass are tallied by degree (the frontier edges Beamer's
    // rule weighs) only while they could reach the bottom-up threshold: a
    // pass claims at most the edges it expands (and at most the scope), and
    // each claim brings at most maxdeg edges.  Bit d of known: the previous
    // pass tallied direction d, so its count is exact.  Whole-GPU policy
    // only: the single-CTA and batched searches are short, and there the
    // extra registers cost more than the gathers they save.
    constexpr bool skip_tally = Ex::nbq > 2;
    unsigned known = 3u;
    const uint32_t dmax32 = skip_tally ? __ldcg(&ex.ctl->maxdeg) : 0u;
    for (unsigned lev = 1;; lev++) {
        const uint32_t nf = last_count(ex, C_FQ), nb = last_count(ex, C_BQ);
        const uint32_t nhf = last_count(ex, C_FH), nhb = last_count(ex, C_BH);
        if (nf + nb + nhf + nhb == 0u) {
            if (last) *last = scope;
            return true;
        }
        if (lev > g.V + 2u) { if (ex.leader()) set_error(ex.ctl, E_NOT_CONVERGED, 40); return false; }
        // Beamer's rule: bottom-up when the frontier has more edges to
        // expand than the scope has vertices to test (times bu_k)
        const uint32_t mf = last_count(ex, C_FE), mb = last_count(ex, C_BE);
        const bool puf = w.bu_k && (unsigned long long)mf > (unsigned long long)scope.n * w.bu_k;
        const bool pub = bw && w.bu_k && (unsigned long long)mb > (unsigned long long)scope.n * w.bu_k;
        unsigned cm = 3u;   // bit d: this pass tallies direction d
        if constexpr (skip_tally) {
            cm = 0u;
            const unsigned long long dmax = dmax32;
#pragma unroll
            for (int d = 0; d < 2; d++) {
                const bool pu = d ? pub : puf;
                const unsigned long long nfd = d ? nb : nf, mfd = d ? mb : mf, nhd = d ? nhb : nhf;
                unsigned long long xe = pu ? scope.n : (((known >> d) & 1u) ? mfd : nfd * dmax) + nhd * CH;
                xe = min(xe, (unsigned long long)scope.n);
                if (w.bu_k && xe * dmax > (unsigned long long)scope.n * w.bu_k) cm |= 1u << d;
            }
            // a bottom-up step may shrink the scope the next pass weighs
            // against, so it tallies both directions (and its finds)
            if (puf || pub) cm = 3u;
            known = cm;
        }
        // bottom-up steps (both directions in one sweep of 64-vertex items)
        // walk the ids instead of the scope list when it holds most of them
        const VList psrc = 2ull * scope.n >= (unsigned long long)g.V ? VList{nullptr, g.V, 1u} : scope;
        const uint32_t nd = (puf || pub) ? (psrc.n + 63u) / 64u : 0u;
        // one shrink per search: a second bottom-up step over the shrunken
        // scope costs more than the top-down steps it would replace
        uint32_t *sout = (Ex::nbq > 2 && (puf || pub) && nshrink == 0u) ? w.S[0] : nullptr;
        ok = run_pass(ex, (puf || pub) ? PH_BFS_PULL : PH_BFS, [&](unsigned, unsigned nxt) {
            const unsigned par = ex.gl & 1u, cp = par ^ 1u;
            // virtual-warp items take VWK groups of frontier vertices
            const uint32_t isz = (lw < 0) ? gsz : (uint32_t)VWK * gsz;
            const uint32_t ngf = (nf + isz - 1u) / isz, ngb = (nb + isz - 1u) / isz;
            const uint32_t items_f = puf ? 0u : nhf + ngf;
            const uint32_t items_b = pub ? 0u : (bw ? nhb + ngb : 0u);
            for (uint32_t it = ex.wid(); it < nd + items_f + items_b; it += ex.nwarps()) {
                if (it < nd) {
                    bfs_pull2(ex, g, w, puf, pub, bw, psrc, it, par, nxt, sout);
                    continue;
                }
                const uint32_t it2 = it - nd;
                const int dir = it2 < items_f ? 0 : 1;
                const uint32_t k = dir ? it2 - items_f : it2;
                const uint32_t nh = dir ? nhb : nhf;
                if (k < nh) {
                    uint2 hc = w.H[dir][cp][k];
                    uint32_t r = w.st[hc.x] & RMASK;
                    auto fn2 = [&](bool v0, uint32_t n0, uint32_t r0, bool v1, uint32_t n1, uint32_t r1) {
                        bfs_edge_visit2(ex, g, w, dir, v0, n0, r0, v1, n1, r1, par, nxt, (cm >> dir) & 1u);
                    };
                    chunk_expand(ex, dir ? g.Br : g.Fr, dir ? g.Bc : g.Fc, hc, r, fn2);
                } else {
                    const uint32_t gi = k - nh;
                    const uint32_t n = dir ? nb : nf;
                    unsigned slot = (lw < 0) ? lane_id() : (lane_id() >> lw);
                    uint32_t i = gi * isz + slot;
                    bool valid = i < n;
                    uint32_t v = valid ? w.Q[dir][cp][i] : 0u;
                    uint32_t r = valid ? (w.st[v] & RMASK) : 0u;
                    bool lead = (lw <= 0) || ((lane_id() & ((1u << lw) - 1u)) == 0u);
                    if (lw < 0) {
                        count_verts(ex, valid && lead);
                        bfs_expand_lanes(ex, g, w, dir, v, valid, r, lw, par, nxt, (cm >> dir) & 1u);
                    } else {
                        uint32_t vk[VWK], rk[VWK];
                        bool ak[VWK];
#pragma unroll
                        for (int j = 0; j < VWK; j++) {
                            const uint32_t ij = i + (uint32_t)j * gsz;
                            ak[j] = ij < n;
                            vk[j] = ak[j] ? w.Q[dir][cp][ij] : 0u;
                        }
#pragma unroll
                        for (int j = 0; j < VWK; j++) {
                            rk[j] = ak[j] ? (w.st[vk[j]] & RMASK) : 0u;
                            count_verts(ex, ak[j] && lead);
                        }
                        bfs_expand_vwk(ex, g, w, dir, vk, ak, rk, lw, par, nxt, (cm >> dir) & 1u);
                    }
                }
            }
            bq_flush(sout ? 3u : 2u, w.qcap, w.Q[0][par], &ex.lc(nxt)[C_FQ], w.Q[1][par],
                     &ex.lc(nxt)[C_BQ], g.V, ex.ctl, &ex.lc(nxt)[C_FE], &ex.lc(nxt)[C_BE], sout,
                     &ex.lc(nxt)[C_SCOPE]);
        });
        if (!ok) return false;
        if (sout) {   // the next bottom-up steps walk the shrunken scope
            scope = VList{sout, last_count(ex, C_SCOPE), 0u};
            nshrink++;
        }
    }
}

// ---------------------------------------------------------------------
// Label propagation over in-edges to a fixpoint:
//   MAXP = true : colour = max id reachable (colorPropagation,
//                 scc_kernels.cu:539-564, pulls the max over out-neighbours)
//   MAXP = false: name = min id reachable (the "WCC" of propagateRange1 /
//                 propagateRange2, scc_kernels.cu:496-536)
// Written as a push over the reverse CSR: when w's value moves, its
// in-neighbours are updated with atomicMax / atomicMin and queued.
// ---------------------------------------------------------------------
template <bool MAXP, class Ex>
__device__ __forceinline__ void prop_visit(Ex &ex, const Graph &g, const Work &w, bool valid, uint32_t u,
                                           uint32_t c, unsigned par, unsigned nxt, uint32_t tag)
{
    bool push = false;
    if (valid) {
        u = guard_id(u, g.V, ex.ctl);
        uint32_t s = w.st[u];
        if (MAXP) {
            if (s < c) push = atomicMax(&w.st[u], c) < c && stamp_claim(w.stamp, u, tag);
        } else {
            if (s != DEAD && s > c) push = atomicMin(&w.st[u], c) > c && stamp_claim(w.stamp, u, tag);
        }
    }
    bq_push(0, push, u, w.qcap, w.Q[0][par], &ex.lc(nxt)[C_FQ], g.V, ex.ctl, 14);
}

template <bool MAXP, class Ex>
__device__ bool ph_propagate(Ex &ex, const Graph &g, const Work &w, VList src0)
{
    uint32_t nq = 0, nh = 0;
    bool first = true;
    for (unsigned lev = 0;; lev++) {
        if (lev > g.V + 2u) { if (ex.leader()) set_error(ex.ctl, E_NOT_CONVERGED, 50); return false; }
        bool ok = run_pass(ex, PH_PROP, [&](unsigned, unsigned nxt) {
            const unsigned par = ex.gl & 1u, cp = par ^ 1u;
            const uint32_t tag = ex.gl + 1u;
            VList src = first ? src0 : VList{w.Q[0][cp], nq, 0u};
            const uint32_t hn = first ? 0u : nh;
            const uint32_t ng = (src.n + 31u) / 32u;
            auto fn = [&](bool valid, uint32_t u, uint32_t c) { prop_visit<MAXP>(ex, g, w, valid, u, c, par, nxt, tag); };
            auto fn2 = [&](bool v0, uint32_t u0, uint32_t c0, bool v1, uint32_t u1, uint32_t c1) {
                prop_visit<MAXP>(ex, g, w, v0, u0, c0, par, nxt, tag);
                prop_visit<MAXP>(ex, g, w, v1, u1, c1, par, nxt, tag);
            };
            for (uint32_t it = ex.wid(); it < hn + ng; it += ex.nwarps()) {
                if (it < hn) {
                    uint2 hc = w.H[0][cp][it];
                    chunk_expand(ex, g.Br, g.Bc, hc, w.st[hc.x] & RMASK, fn2);
                } else {
                    uint32_t i = (it - hn) * 32u + lane_id();
                    bool valid = i < src.n;
                    uint32_t v = valid ? src.at(i) : 0u;
                    uint32_t c = valid ? (w.st[v] & RMASK) : 0u;
                    if (!MAXP && valid && c != v) {
                        // pointer jumping: the name of v's name is also reachable from v
                        // (the same fixpoint, reached in fewer sweeps on long chains)
                        const uint32_t s2 = w.st[c];
                        if (s2 != DEAD && (s2 & RMASK) < c) {
                            c = s2 & RMASK;
                            atomicMin(&w.st[v], c);
                        }
                    }
                    uint32_t beg = 0, deg = 0;
                    if (valid) { beg = __ldg(&g.Br[v]); deg = __ldg(&g.Br[v + 1]) - beg; }
                    bool heavy = deg > HEAVY_T;
                    warp_push_chunks(v, heavy ? (deg + CH - 1u) / CH : 0u, w.H[0][par],
                                     &ex.lc(nxt)[C_FH], w.hcap, ex.ctl);
                    if (heavy) deg = 0u;
                    count_verts(ex, valid);
                    count_edges(ex, lbs_expand(beg, deg, c, g.Bc, fn));
                }
            }
            bq_flush(1, w.qcap, w.Q[0][par], &ex.lc(nxt)[C_FQ], nullptr, nullptr, g.V, ex.ctl);
        });
        if (!ok) return false;
        first = false;
        nq = last_count(ex, C_FQ);
        nh = last_count(ex, C_FH);
        if (nq + nh == 0u) return true;
    }
}

// ---------------------------------------------------------------------
// Hong update (scc_kernels.cu:124-142): FV and BV -> the SCC of the range's
// pivot; otherwise the vertex moves to one of three fresh sub-range names
// and is appended to the next live list.  With fold, the survivors also
// bid for the pivot of their new range, which replaces the reference's
// separate pollForPivots/selectPivots launches (scc_WCC.cu:860-862).
// ---------------------------------------------------------------------
template <class Ex>
__device__ bool ph_hong_update(Ex &ex, const Graph &g, const Work &w, VList src, uint32_t *Lout,
                               bool single, bool fold)
{
    return run_pass(ex, PH_HONG_UPDATE, [&](unsigned, unsigned nxt) {
        uint32_t mn = 0xFFFFFFFFu;   // single: smallest member of the pivot's SCC seen by this thread
        for (uint32_t base = ex.wid() * 128u; base < src.n; base += ex.nwarps() * 128u) {
            uint32_t v[4], s[4];
            bool ok[4];
            load_list4(src, base + 4u * lane_id(), v, ok);
#pragma unroll
            for (int j = 0; j < 4; j++) s[j] = ok[j] ? w.st[v[j]] : DEAD;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                bool surv = false, scc = false;
                uint32_t p = 0u, nr = 0u;
                if (s[j] != DEAD) {
                    p = key_vertex(w.pivkey[single ? 0u : (s[j] & RMASK)]);
                    if ((s[j] & FVB) && (s[j] & BVB)) {
                        w.st[v[j]] = DEAD;
                        w.label[v[j]] = p;
                        scc = true;
                    } else {
                        nr = split_name(g.V, p, s[j]);
                        w.st[v[j]] = nr;
                        surv = true;
                    }
                }
                if (single) mn = scc ? min(mn, v[j]) : mn;
                else smin_fold(scc, p, v[j], w.smin);
                bq_add_edges(0, surv ? __ldg(&g.Fr[v[j] + 1u]) - __ldg(&g.Fr[v[j]]) : 0u);
                bq_push(0, surv, v[j], w.qcap, Lout, &ex.lc(nxt)[C_LIST], g.V, ex.ctl, 15);
                if (fold) {
                    // the new ranges are listed by their first bid (as in ph_pivots)
                    const bool first = range_max_atomic(surv, nr, surv ? pivot_key(g, v[j]) : 0ull, w.pivkey);
                    warp_push(first, nr, w.Q[0][ex.gl & 1u], &ex.lc(nxt)[C_RNG], g.V + 1u, ex.ctl, 22);
                }
            }
            count_verts_n(ex, (unsigned)ok[0] + ok[1] + ok[2] + ok[3]);
        }
        if (single) block_min_atomic(mn, w.pivkey[0] ? &w.smin[key_vertex(w.pivkey[0])] : w.smin);
        bq_flush(1, w.qcap, Lout, &ex.lc(nxt)[C_LIST], nullptr, nullptr, g.V, ex.ctl, &ex.lc(nxt)[C_FE]);
    });
}

// Slota: the first FW-BW's SCC is final; every other live vertex starts
// the colouring with colour = its own id (assignUniqueRange,
// scc_kernels.cu:477-484) and is appended to the live list.
template <class Ex>
__device__ bool ph_slota_first_update(Ex &ex, const Graph &g, const Work &w, VList src, uint32_t *Lout)
{
    return run_pass(ex, PH_SLOTA_FIRST_UPDATE, [&](unsigned, unsigned nxt) {
        const uint32_t p = key_vertex(w.pivkey[0]);
        uint32_t mn = 0xFFFFFFFFu;   // smallest member of p's SCC seen by this thread
        for (uint32_t base = ex.wid() * 128u; base < src.n; base += ex.nwarps() * 128u) {
            uint32_t v[4], s[4];
            bool ok[4];
            load_list4(src, base + 4u * lane_id(), v, ok);
#pragma unroll
            for (int j = 0; j < 4; j++) s[j] = ok[j] ? w.st[v[j]] : DEAD;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                bool surv = false, scc = false;
                if (s[j] != DEAD) {
                    if ((s[j] & FVB) && (s[j] & BVB)) { w.st[v[j]] = DEAD; w.label[v[j]] = p; scc = true; }
                    else { w.st[v[j]] = v[j]; w.stamp[v[j]] = 0u; surv = true; }   // the colouring's work lists stamp them
                }
                mn = scc ? min(mn, v[j]) : mn;
                bq_add_edges(0, surv ? __ldg(&g.Fr[v[j] + 1u]) - __ldg(&g.Fr[v[j]]) : 0u);
                bq_push(0, surv, v[j], w.qcap, Lout, &ex.lc(nxt)[C_LIST], g.V, ex.ctl, 16);
            }
            count_verts_n(ex, (unsigned)ok[0] + ok[1] + ok[2] + ok[3]);
        }
        block_min_atomic(mn, w.pivkey[0] ? &w.smin[p] : w.smin);   // mn stays 0xFFFFFFFF without a pivot
        bq_flush(1, w.qcap, Lout, &ex.lc(nxt)[C_LIST], nullptr, nullptr, g.V, ex.ctl, &ex.lc(nxt)[C_FE]);
    });
}

// The same update on the whole-GPU policy, where the search kept a
// shrinking scope: members of the first SCC (both visited bits) keep that
// mark as their state -- no later phase treats it as live, and the label
// write maps it to the SCC's smallest member, Ctl::first_min, which every
// CTA folds in here from the completions it saw -- so only the search's
// final scope is walked, not every vertex the search could reach.
template <class Ex>
__device__ bool ph_slota_first_update_lazy(Ex &ex, const Graph &g, const Work &w, VList src, uint32_t *Lout)
{
    return run_pass(ex, PH_SLOTA_FIRST_UPDATE, [&](unsigned, unsigned nxt) {
        for (uint32_t base = ex.wid() * 128u; base < src.n; base += ex.nwarps() * 128u) {
            uint32_t v[4], s[4];
            bool ok[4];
            load_list4(src, base + 4u * lane_id(), v, ok);
#pragma unroll
            for (int j = 0; j < 4; j++) s[j] = ok[j] ? w.st[v[j]] : DEAD;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const bool surv = s[j] != DEAD && (s[j] & (FVB | BVB)) != (FVB | BVB);
                if (surv) { w.st[v[j]] = v[j]; w.stamp[v[j]] = 0u; }
                bq_add_edges(0, surv ? __ldg(&g.Fr[v[j] + 1u]) - __ldg(&g.Fr[v[j]]) : 0u);
                bq_push(0, surv, v[j], w.qcap, Lout, &ex.lc(nxt)[C_LIST], g.V, ex.ctl, 16);
            }
            count_verts_n(ex, (unsigned)ok[0] + ok[1] + ok[2] + ok[3]);
        }
        __syncthreads();
        if (threadIdx.x == 0 && *cta_first_min() != 0xFFFFFFFFu) atomicMin(&ex.ctl->first_min, *cta_first_min());
        bq_flush(1, w.qcap, Lout, &ex.lc(nxt)[C_LIST], nullptr, nullptr, g.V, ex.ctl, &ex.lc(nxt)[C_FE]);
    });
}

// Slota peel end (updateColoring, scc_kernels.cu:614-623; fwdColoring's
// rangeSet, :607): visited vertices belong to their root's SCC; the rest
// restart from their own colour and form the next live list.
template <class Ex>
__device__ bool ph_slota_peel_update(Ex &ex, const Graph &g, const Work &w, VList src, uint32_t *Lout)
{
    return run_pass(ex, PH_SLOTA_PEEL_UPDATE, [&](unsigned, unsigned nxt) {
        for (uint32_t base = ex.wid() * 128u; base < src.n; base += ex.nwarps() * 128u) {
            uint32_t v[4], s[4];
            bool ok[4];
            load_list4(src, base + 4u * lane_id(), v, ok);
#pragma unroll
            for (int j = 0; j < 4; j++) s[j] = ok[j] ? w.st[v[j]] : 0u;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                bool surv = false, scc = false;
                uint32_t c = 0u;
                if (ok[j]) {
                    if (s[j] & FVB) { c = s[j] & RMASK; w.st[v[j]] = DEAD; w.label[v[j]] = c; scc = true; }
                    else { w.st[v[j]] = v[j]; surv = true; }
                }
                smin_fold(scc, c, v[j], w.smin);
                bq_add_edges(0, surv ? __ldg(&g.Fr[v[j] + 1u]) - __ldg(&g.Fr[v[j]]) : 0u);
                bq_push(0, surv, v[j], w.qcap, Lout, &ex.lc(nxt)[C_LIST], g.V, ex.ctl, 17);
            }
            count_verts_n(ex, (unsigned)ok[0] + ok[1] + ok[2] + ok[3]);
        }
        bq_flush(1, w.qcap, Lout, &ex.lc(nxt)[C_LIST], nullptr, nullptr, g.V, ex.ctl, &ex.lc(nxt)[C_FE]);
    });
}

// Hong: compact the live list and give every live vertex its own id as
// name (assignUniqueRange, scc_kernels.cu:477-484) before the min-label
// propagation.
template <class Ex>
__device__ bool ph_compact_rename(Ex &ex, const Graph &g, const Work &w, VList src, uint32_t *Lout)
{
    return run_pass(ex, PH_RENAME, [&](unsigned, unsigned nxt) {
        for (uint32_t base = ex.wid() * 128u; base < src.n; base += ex.nwarps() * 128u) {
            uint32_t v[4], s[4];
            bool ok[4];
            load_list4(src, base + 4u * lane_id(), v, ok);
#pragma unroll
            for (int j = 0; j < 4; j++) s[j] = ok[j] ? w.st[v[j]] : DEAD;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const bool surv = s[j] != DEAD;
                if (surv) w.st[v[j]] = v[j];
                bq_push(0, surv, v[j], w.qcap, Lout, &ex.lc(nxt)[C_LIST], g.V, ex.ctl, 18);
            }
            count_verts_n(ex, (unsigned)ok[0] + ok[1] + ok[2] + ok[3]);
        }
        bq_flush(1, w.qcap, Lout, &ex.lc(nxt)[C_LIST], nullptr, nullptr, g.V, ex.ctl);
    });
}

// Per-range pivot bids over a list (pollForPivots, scc_kernels.cu:57-74).
template <class Ex>
__device__ bool ph_pivots(Ex &ex, const Graph &g, const Work &w, VList src)
{
    // every range is listed once, by its first bid, in Q[0][parity of this
    // pass]: the next pass seeds the pivots from that list
    return run_pass(ex, PH_PIVOTS, [&](unsigned, unsigned nxt) {
        const unsigned par = ex.gl & 1u;
        for (uint32_t base = ex.wid() * 32u; base < src.n; base += ex.nwarps() * 32u) {
            uint32_t i = base + lane_id();
            bool valid = i < src.n;
            uint32_t v = valid ? src.at(i) : 0u;
            uint32_t r = valid ? (w.st[v] & RMASK) : 0u;
            const bool first = range_max_atomic(valid, r, valid ? pivot_key(g, v) : 0ull, w.pivkey);
            warp_push(first, r, w.Q[0][par], &ex.lc(nxt)[C_RNG], g.V + 1u, ex.ctl, 21);
            bq_add_edges(0, valid ? __ldg(&g.Fr[v + 1u]) - __ldg(&g.Fr[v]) : 0u);
        }
        bq_flush_edges(&ex.lc(nxt)[C_FE]);   // out-arcs of the live list (the residual check)
    });
}

// ---------------------------------------------------------------------
// drivers
// ---------------------------------------------------------------------
struct Carry {
    unsigned gl;
    unsigned lsel;
    uint32_t nL;
    uint32_t nR;    // Hong: ranges listed by the last bidding pass (in Q[0][its parity])
    uint32_t nE;    // out-arcs of the live vertices (tallied by the pass that listed them)
};

enum { RUN_DONE = 0, RUN_SWITCH = 1, RUN_RESIDUAL = 2, RUN_ERROR = -1 };

// ---------------------------------------------------------------------
// Small residuals: when the live vertices left for the main loop / the
// colouring peels are few (at most RES_MAX_V, with at most RES_MAX_E
// out-arcs), their SCCs are found on one CTA in shared memory instead of
// by further whole-GPU passes.  SCCs never contain a vertex whose SCC is
// already known, so the SCCs of the live vertices are those of the
// subgraph they induce; every SCC found here counts as a pivot SCC, as the
// reference counts each SCC its main loop / colouring finds once
// (scc_WCC.cu:933-949, scc_Coloring.cu:640-652), so the counters and the
// canonical labels are those of any complete run.
//   pass 1 (all CTAs): live vertex L[i] gets the state word FV|BV|(i + 1)
//          (at a loop head the only other vertices with both bits are the
//          first SCC's members, marked FV|BV|0);
//   pass 2 (all CTAs): the arcs between live vertices, as (i << 16) | j,
//          into a work queue;
//   then one CTA loads them into shared memory and peels SCCs by colour
//   propagation (max of the local ids reachable on even peels, min on odd
//   ones, so a chain is cut from either end) and a forward search inside
//   each colour from its root, as scc_Coloring.cu:590-637 does, but with
//   __syncthreads barriers between sweeps.
// ---------------------------------------------------------------------
constexpr uint32_t RES_MAX_V = 4096;
constexpr uint32_t RES_MAX_E = 16384;

__host__ __device__ __forceinline__ uint32_t res_al4(uint32_t x) { return (x + 3u) & ~3u; }
// shared memory of the solver: gid, off, aux (u32), col (u16), flag (u8), adj (u16)
__host__ __device__ __forceinline__ uint32_t res_smem_bytes(uint32_t n, uint32_t m)
{
    return 4u * n + 4u * (n + 1u) + 4u * n + res_al4(2u * n) + res_al4(n) + res_al4(2u * m);
}

// Uniform decision (same in every thread of the launch or CTA): solve the
// live list on one CTA?  The solver uses the staging queues' shared memory.
template <class Ex>
__device__ __forceinline__ bool res_fits(const Graph &g, const Work &w, const Carry &cy)
{
    if (Ex::cluster || cy.nL == 0u || cy.nL > RES_MAX_V || cy.nE > RES_MAX_E || cy.nE > g.V + 1u) return false;
    const uint32_t avail = Ex::nbq * (blockDim.x >> 5) * w.qcap * 4u;
    return res_smem_bytes(cy.nL, cy.nE) <= avail;
}

// Block-wide exclusive prefix sum of a[0..len) in place (shared memory).
// Every thread of the CTA calls it.
__device__ __forceinline__ void block_excl_scan(uint32_t *a, uint32_t len)
{
    __shared__ uint32_t s_part[32];
    const uint32_t per = (len + blockDim.x - 1u) / blockDim.x;
    const uint32_t lo = threadIdx.x * per, hi = min(lo + per, len);
    uint32_t sum = 0;
    for (uint32_t i = lo; i < hi; i++) sum += a[i];
    const uint32_t incl = warp_incl_scan(sum);
    const unsigned wi = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane_id() == 31u) s_part[wi] = incl;
    __syncthreads();
    if (wi == 0) {
        const uint32_t x = lane_id() < nw ? s_part[lane_id()] : 0u;
        const uint32_t xs = warp_incl_scan(x);
        if (lane_id() < nw) s_part[lane_id()] = xs - x;   // exclusive offset of each warp
    }
    __syncthreads();
    uint32_t run = s_part[wi] + incl - sum;
    for (uint32_t i = lo; i < hi; i++) {
        const uint32_t x = a[i];
        a[i] = run;
        run += x;
    }
    __syncthreads();
}

// Passes 1 and 2 (every CTA of the policy).  On return the arcs are in
// Q[1][(cy.gl - 1) & 1] and their number in the pass counter C_BQ.
template <class Ex>
__device__ bool res_extract(Ex &ex, const Graph &g, const Work &w, Carry &cy)
{
    const uint32_t *L = w.L[cy.lsel];
    const uint32_t n = cy.nL;
    if (!run_pass(ex, PH_RES_TAG, [&](unsigned, unsigned) {
            for (uint32_t i = ex.tid(); i < n; i += ex.nthr()) w.st[L[i]] = FVB | BVB | (i + 1u);
        }))
        return false;
    const bool ok = run_pass(ex, PH_RES_EXTRACT, [&](unsigned, unsigned nxt) {
        uint32_t *eb = w.Q[1][ex.gl & 1u];
        for (uint32_t base = ex.wid() * 32u; base < n; base += ex.nwarps() * 32u) {
            const uint32_t i = base + lane_id();
            const bool valid = i < n;
            const uint32_t v = valid ? L[i] : 0u;
            const uint32_t beg = valid ? __ldg(&g.Fr[v]) : 0u, deg = valid ? __ldg(&g.Fr[v + 1u]) - beg : 0u;
            auto fn = [&](bool ok2, uint32_t u, uint32_t src) {
                bool hit = false;
                uint32_t e = 0;
                if (ok2) {
                    const uint32_t s = w.st[guard_id(u, g.V, ex.ctl)];
                    // live vertex i carries FV|BV|(i + 1); FV|BV|0 marks the first SCC's members
                    hit = (s & (FVB | BVB)) == (FVB | BVB) && (s & RMASK) != 0u;
                    e = (src << 16) | ((s & RMASK) - 1u);
                }
                warp_push(hit, e, eb, &ex.lc(nxt)[C_BQ], RES_MAX_E, ex.ctl, 24);
            };
            count_edges(ex, lbs_expand(beg, deg, i, g.Fc, fn));
        }
    });
    cy.gl = ex.gl;
    return ok;
}

// The solver (every thread of one CTA).  L[0..n): the live vertices;
// eb[0..m): their arcs (i << 16) | j.  Writes every live vertex's
// canonical label (LBL_SELF: the smallest id of its SCC) and DEAD state, and
// adds the SCCs found to n_pivot.  Each peel removes at least the root with
// the largest (or smallest) key, so at most n peels, each with at most n + 1
// sweeps per fixpoint.
// With out set the canonical labels of the residual vertices go straight to
// out and their state words keep the residual tag: the other CTAs are
// writing every other vertex's label meanwhile, deciding by that tag.
static __device__ __noinline__ void res_solve(const Graph &g, const Work &w, const uint32_t *L, uint32_t n, const uint32_t *eb,
                          uint32_t m, Ctl *ctl, uint32_t *out = nullptr)
{
    constexpr uint8_t ALIVE = 1, VIS = 2;
    char *sb = reinterpret_cast<char *>(&sccb_dsmem[BQ_HDR]);
    uint32_t *gid = reinterpret_cast<uint32_t *>(sb);
    uint32_t *off = gid + n;
    uint32_t *aux = off + n + 1u;                  // fill cursor, then smallest member id per root
    uint16_t *col = reinterpret_cast<uint16_t *>(aux + n);
    uint8_t *flag = reinterpret_cast<uint8_t *>(sb + 12u * n + 4u + res_al4(2u * n));
    uint16_t *adj = reinterpret_cast<uint16_t *>(sb + 12u * n + 4u + res_al4(2u * n) + res_al4(n));
    __shared__ uint32_t s_alive, s_npiv, s_peels;
    const uint32_t t = threadIdx.x, T = blockDim.x;
    for (uint32_t i = t; i < n; i += T) {
        gid[i] = L[i];
        off[i] = 0u;
        flag[i] = ALIVE;
    }
    if (t == 0) { off[n] = 0u; s_alive = n; s_npiv = 0u; s_peels = 0u; }
    __syncthreads();
    for (uint32_t k = t; k < m; k += T) atomicAdd(&off[eb[k] >> 16], 1u);
    __syncthreads();
    block_excl_scan(off, n + 1u);
    for (uint32_t i = t; i < n; i += T) aux[i] = off[i];
    __syncthreads();
    for (uint32_t k = t; k < m; k += T) {
        const uint32_t e = eb[k];
        adj[atomicAdd(&aux[e >> 16], 1u)] = (uint16_t)(e & 0xFFFFu);
    }
    __syncthreads();
    for (uint32_t i = t; i < n; i += T) aux[i] = 0xFFFFFFFFu;
    __syncthreads();
    bool failed = false;
    for (uint32_t peel = 0;; peel++) {
        if (s_alive == 0u) break;
        if (peel > n + 1u) { failed = true; break; }
        const bool up = (peel & 1u) == 0u;
        for (uint32_t i = t; i < n; i += T)
            if (flag[i] & ALIVE) col[i] = (uint16_t)(up ? i : n - 1u - i);
        __syncthreads();
        // colour = largest key reachable (scc_kernels.cu:539-564)
        for (uint32_t sweep = 0;; sweep++) {
            int ch = 0;
            for (uint32_t i = t; i < n; i += T) {
                if (!(flag[i] & ALIVE)) continue;
                uint16_t c = col[i];
                for (uint32_t e = off[i]; e < off[i + 1u]; e++) {
                    const uint16_t j = adj[e];
                    if ((flag[j] & ALIVE) && col[j] > c) c = col[j];
                }
                if (c > col[i]) { col[i] = c; ch = 1; }
            }
            if (!__syncthreads_or(ch)) break;
            if (sweep > n + 1u) { failed = true; break; }
        }
        if (failed) break;
        // roots keep their own key; the forward search inside each colour
        // (scc_kernels.cu:567-610) marks their SCCs
        for (uint32_t i = t; i < n; i += T)
            if ((flag[i] & ALIVE) && col[i] == (up ? i : n - 1u - i)) flag[i] |= VIS;
        __syncthreads();
        for (uint32_t sweep = 0;; sweep++) {
            int ch = 0;
            for (uint32_t i = t; i < n; i += T) {
                if ((flag[i] & (ALIVE | VIS)) != (ALIVE | VIS)) continue;
                for (uint32_t e = off[i]; e < off[i + 1u]; e++) {
                    const uint16_t j = adj[e];
                    if ((flag[j] & (ALIVE | VIS)) == ALIVE && col[j] == col[i]) { flag[j] |= VIS; ch = 1; }
                }
            }
            if (!__syncthreads_or(ch)) break;
            if (sweep > n + 1u) { failed = true; break; }
        }
        if (failed) break;
        uint32_t done = 0, roots = 0;
        for (uint32_t i = t; i < n; i += T) {
            if ((flag[i] & (ALIVE | VIS)) != (ALIVE | VIS)) continue;
            const uint32_t r = up ? col[i] : n - 1u - col[i];
            atomicMin(&aux[r], gid[i]);
            col[i] = (uint16_t)r;   // the root, from here on
            flag[i] = 0;
            done++;
            roots += (r == i) ? 1u : 0u;
        }
        done = __reduce_add_sync(FULL, done);
        roots = __reduce_add_sync(FULL, roots);
        if (lane_id() == 0 && done) { atomicSub(&s_alive, done); atomicAdd(&s_npiv, roots); }
        if (t == 0) s_peels = peel + 1u;
        __syncthreads();
    }
    if (failed) {
        if (t == 0) set_error(ctl, E_NOT_CONVERGED, 71);
        return;
    }
    for (uint32_t i = t; i < n; i += T) {
        w.label[gid[i]] = LBL_SELF | aux[col[i]];
        if (out) out[gid[i] - 1u] = aux[col[i]];
        else w.st[gid[i]] = DEAD;
    }
    if (t == 0) {
        atomicAdd(&ctl->n_pivot, (unsigned long long)s_npiv);
        atomicAdd(&ctl->outer, s_peels);
    }
    __syncthreads();
}

// Records the solver as one more pass in the pass trace (one CTA).
__device__ __forceinline__ void res_trace(Ctl *ctl, unsigned gl, uint32_t n)
{
    if (threadIdx.x == 0 && ctl->trace && gl < ctl->trace_cap) {
        ctl->trace[2 * gl] = gtimer();
        ctl->trace[2 * gl + 1] = (unsigned long long)PH_RES_SOLVE | ((unsigned long long)n << 8);
    }
}

// Residual path at a main-loop / peel head.  On the whole-GPU policy it
// returns RUN_RESIDUAL after the two passes (CTA 0 then solves and the
// others leave); on one CTA it also solves and returns RUN_DONE.
template <class Ex>
__device__ int residual(Ex &ex, const Graph &g, const Work &w, Carry &cy)
{
    if (!res_extract(ex, g, w, cy)) return RUN_ERROR;
    if (Ex::grid) return RUN_RESIDUAL;
    res_solve(g, w, w.L[cy.lsel], cy.nL, w.Q[1][(cy.gl - 1u) & 1u], last_count(ex, C_BQ), ex.ctl);
    res_trace(ex.ctl, ex.gl, cy.nL);
    ex.gl++;
    cy.gl = ex.gl;
    cy.nL = 0u;
    return ex.sync() ? RUN_DONE : RUN_ERROR;
}

// Hong main loop (scc_WCC.cu:851-930): per-range pivots, FW-BW, update,
// until no vertex is left.  Entry: live list L[lsel] with nL entries and
// the pivot bids of their ranges already in pivkey.
template <class Ex>
__device__ int hong_loop(Ex &ex, const Graph &g, const Work &w, Carry &cy, uint32_t tail_n)
{
    while (cy.nL > 0u) {
        if (res_fits<Ex>(g, w, cy)) return residual(ex, g, w, cy);
        if (Ex::grid && cy.nL <= tail_n) { cy.gl = ex.gl; return RUN_SWITCH; }
        if (ex.leader()) ex.ctl->outer++;
        const VList L{w.L[cy.lsel], cy.nL, 0u};
        const VList R{w.Q[0][(ex.gl & 1u) ^ 1u], cy.nR, 0u};   // written by the previous pass
        if (!ph_bfs(ex, g, w, R, SeedRanges{}, true, -1, L)) return RUN_ERROR;
        if (!ph_hong_update(ex, g, w, L, w.L[cy.lsel ^ 1u], false, true)) return RUN_ERROR;
        cy.nL = last_count(ex, C_LIST);
        cy.nR = last_count(ex, C_RNG);
        cy.nE = last_count(ex, C_FE);
        cy.lsel ^= 1u;
        cy.gl = ex.gl;
    }
    return RUN_DONE;
}

// First pivot over the live vertices after trim1 to fixpoint
// (pollForFirstPivot / selectFirstPivot, scc_WCC.cu:701-703); the live
// vertices are compacted into Lout on the way.
template <class Ex>
__device__ bool ph_first_pivot(Ex &ex, const Graph &g, const Work &w, uint32_t *Lout)
{
    return run_pass(ex, PH_FIRST_PIVOT, [&](unsigned, unsigned nxt) {
        unsigned long long best = 0;
        for (uint32_t base = ex.wid() * 128u; base <= g.V; base += ex.nwarps() * 128u) {
            const uint32_t i0 = base + 4u * lane_id();
            uint32_t st4[4] = {DEAD, DEAD, DEAD, DEAD};
            if (i0 + 3u <= g.V) {
                const uint4 x = *reinterpret_cast<const uint4 *>(w.st + i0);
                st4[0] = x.x; st4[1] = x.y; st4[2] = x.z; st4[3] = x.w;
            } else {
                for (uint32_t j = 0; j < 4u && i0 + j <= g.V; j++) st4[j] = w.st[i0 + j];
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint32_t v = i0 + (uint32_t)j;
                const bool live = v >= 1u && v <= g.V && st4[j] != DEAD;
                if (live) {
                    unsigned long long k = pivot_key(g, v);
                    best = k > best ? k : best;
                }
                bq_push(0, live, v, w.qcap, Lout, &ex.lc(nxt)[C_LIST], g.V, ex.ctl, 20);
            }
            count_verts_n(ex, i0 <= g.V ? min(4u, g.V + 1u - i0) : 0u);
        }
        block_max_atomic(best, &w.pivkey[0]);
        bq_flush(1, w.qcap, Lout, &ex.lc(nxt)[C_LIST], nullptr, nullptr, g.V, ex.ctl);
    });
}

__device__ __forceinline__ unsigned long long vld64(const unsigned long long *p)
{
    return *(const volatile unsigned long long *)p;
}

// The first FW-BW of every driver, from the single pivot in pivkey[0]
// (scc_WCC.cu:717-743, scc_Coloring.cu:539-565; wHong / wSlota run it with
// the virtual-warp schedule, scc_WCC.cu:209-317, scc_Coloring.cu:154-263).
template <class Ex>
__device__ bool first_fwbw(Ex &ex, const Graph &g, const Work &w, int lw, VList scope, VList *last = nullptr)
{
    const unsigned long long k = vld64(&w.pivkey[0]);
    const uint32_t p = k ? key_vertex(k) : 0u;
    return ph_bfs(ex, g, w, VList{nullptr, k ? 1u : 0u, p}, SeedOne{p}, true, lw, scope, last);
}

// vHong / wHong up to the main loop (scc_WCC.cu:573-848): trim1*, first
// pivot, FW-BW, update, trim1*, trim2, trim1*, "WCC", first per-range pivots.
template <class Ex>
__device__ int hong_front(Ex &ex, const Graph &g, const Work &w, bool t1, bool t2, int lw, Carry &cy)
{
    const VList all{nullptr, g.V, 1u};
    VList scope = all;
    if (!ph_init(ex, g, w, !t1)) return RUN_ERROR;
    if (t1) {
        if (!ph_trim1_fix(ex, g, w, all, true)) return RUN_ERROR;
        if (!ph_first_pivot(ex, g, w, w.L[0])) return RUN_ERROR;
        scope = VList{w.L[0], last_count(ex, C_LIST), 0u};
    }
    if (!first_fwbw(ex, g, w, lw, scope)) return RUN_ERROR;
    if (!ph_hong_update(ex, g, w, scope, w.L[1], true, false)) return RUN_ERROR;
    const VList L1{w.L[1], last_count(ex, C_LIST), 0u};
    if (t1 && !ph_trim1_fix(ex, g, w, L1, false)) return RUN_ERROR;
    if (t2 && !ph_trim2(ex, g, w, L1)) return RUN_ERROR;
    if (t1 && t2 && !ph_trim1_fix(ex, g, w, L1, false)) return RUN_ERROR;
    if (!ph_compact_rename(ex, g, w, L1, w.L[0])) return RUN_ERROR;
    cy.lsel = 0u;
    cy.nL = last_count(ex, C_LIST);
    const VList L{w.L[0], cy.nL, 0u};
    if (!ph_propagate<false>(ex, g, w, L)) return RUN_ERROR;
    if (!ph_pivots(ex, g, w, L)) return RUN_ERROR;
    cy.nR = last_count(ex, C_RNG);
    cy.nE = last_count(ex, C_FE);
    cy.gl = ex.gl;
    return RUN_DONE;
}

// vSlota / wSlota up to the colouring loop (scc_Coloring.cu:403-587):
// trim1 once, first pivot, FW-BW, update.  t2 is not used by the
// reference's Slota drivers.
template <class Ex>
__device__ int slota_front(Ex &ex, const Graph &g, const Work &w, bool t1, int lw, Carry &cy)
{
    VList scope{nullptr, g.V, 1u};
    if (t1) {
        if (!ph_init_trim1(ex, g, w, w.L[0])) return RUN_ERROR;
        scope = VList{w.L[0], last_count(ex, C_LIST), 0u};
    } else if (!ph_init(ex, g, w, true)) {
        return RUN_ERROR;
    }
    if constexpr (Ex::nbq > 2) {
        // whole GPU: the first SCC's members keep their FV|BV mark and the
        // update walks only the search's final, shrunken scope
        VList last = scope;
        if (!first_fwbw(ex, g, w, lw, scope, &last)) return RUN_ERROR;
        if (!ph_slota_first_update_lazy(ex, g, w, last, w.L[1])) return RUN_ERROR;
    } else {
        if (!first_fwbw(ex, g, w, lw, scope)) return RUN_ERROR;
        if (!ph_slota_first_update(ex, g, w, scope, w.L[1])) return RUN_ERROR;
    }
    cy.lsel = 1u;
    cy.nL = last_count(ex, C_LIST);
    cy.nE = last_count(ex, C_FE);
    cy.gl = ex.gl;
    return RUN_DONE;
}

// Colouring peels (scc_Coloring.cu:590-637): max-colour propagation, roots
// colour == id, forward reachability inside the colour, update.
template <class Ex>
__device__ int slota_peels(Ex &ex, const Graph &g, const Work &w, Carry &cy, uint32_t tail_n)
{
    while (cy.nL > 0u) {
        if (res_fits<Ex>(g, w, cy)) return residual(ex, g, w, cy);
        if (Ex::grid && cy.nL <= tail_n) { cy.gl = ex.gl; return RUN_SWITCH; }
        if (ex.leader()) ex.ctl->outer++;
        const VList L{w.L[cy.lsel], cy.nL, 0u};
        if (!ph_propagate<true>(ex, g, w, L)) return RUN_ERROR;
        if (!ph_bfs(ex, g, w, L, SeedRoot{}, false, -1, L)) return RUN_ERROR;
        if (!ph_slota_peel_update(ex, g, w, L, w.L[cy.lsel ^ 1u])) return RUN_ERROR;
        cy.nL = last_count(ex, C_LIST);
        cy.nE = last_count(ex, C_FE);
        cy.lsel ^= 1u;
        cy.gl = ex.gl;
    }
    return RUN_DONE;
}

}  // namespace sccb
