// Device-side building blocks of the B200 SCC engine.
//
// Vertex state is one 32-bit word per vertex (st[v]):
//   bits  0..29  range name (FW-BW subproblem, Hong) or colour (Slota);
//                0x3FFFFFFF marks a vertex whose SCC is already known
//                (the reference's rangeSet tag, include/scc.h:36-37)
//   bit   30     forward-visited  (FV, include/scc.h:24)
//   bit   31     backward-visited (BV, include/scc.h:26)
// so one gather per adjacency entry tells whether the neighbour is live, in
// the same subproblem and unvisited.  The reference keeps uint8 tags plus a
// uint32 range and reads both per edge (scc_kernels.cu:374-377).
//
// Every phase is written once against an execution policy:
//   GridExec   all CTAs of a cooperative (co-resident) launch; passes end in
//              a grid barrier whose wait is bounded by %globaltimer;
//   BlockExec  one CTA; passes end in __syncthreads.
// The plain path runs GridExec and drops to BlockExec on CTA 0 when the live
// set gets small; the batched form runs one BlockExec per graph.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sccb {

constexpr uint32_t RMASK = 0x3FFFFFFFu;
constexpr uint32_t DEAD = 0x3FFFFFFFu;
constexpr uint32_t FVB = 0x40000000u;
constexpr uint32_t BVB = 0x80000000u;
constexpr uint32_t FULL = 0xFFFFFFFFu;
constexpr uint32_t MAX_V = 0x0FFFFFFEu;   // 4V+3 split names must stay below DEAD
// label[v] with this bit set holds v's canonical label itself (the low
// bits): a vertex that is its own SCC (trim-1, trim-2, small residual SCCs)
// needs no smin entry and no gather when the labels are written out.
constexpr uint32_t LBL_SELF = 0x80000000u;

// Load-balancing constants of the frontier expansion: a frontier vertex
// whose degree exceeds HEAVY_T is cut into CH-edge chunks that the next pass
// spreads over all warps.
constexpr uint32_t HEAVY_T = 256;
constexpr uint32_t CH = 512;

// error codes shared with the host (include/scc_b200.h)
constexpr int E_OVERFLOW = 20;
constexpr int E_NOT_CONVERGED = 21;
constexpr int E_TIMEOUT = 22;
constexpr int E_BAD_GRAPH = 23;

enum { C_FQ = 0, C_BQ = 1, C_FH = 2, C_BH = 3, C_LIST = 4, C_FE = 5, C_BE = 6, C_RNG = 7, C_SCOPE = 8, NCNT = 9 };

struct __align__(128) Ctl {
    // grid barrier arrival counter and the sticky error code share one
    // 8-byte word so that a waiter polls both with one load
    unsigned bar_count;
    int error;
    int where; unsigned _p0[29];
    unsigned lc[3][NCNT];                          // per-pass counters, 3-slot ring
    unsigned maxdeg;                               // largest out- or in-degree (init sweep)
    unsigned _p3[4];
    unsigned long long n_trim1, n_trim2, n_pivot;
    unsigned long long t_edges, t_verts;           // instrumented work counters
    unsigned passes, outer;                        // passes run, peels / iterations
    unsigned long long timeout_ns;
    unsigned tail_pass;                            // pass at which CTA 0 took over (0 = never)
    unsigned nlive_tail;
    unsigned long long t_start;                    // %globaltimer at kernel entry
    unsigned long long *trace;                     // optional: 2 words per pass
    unsigned trace_cap;
    unsigned labels_done;                          // the SCC kernel wrote the canonical labels itself
    unsigned first_min;                            // smallest member of the first pivot's SCC when its members
                                                   // keep the FV|BV mark (lazy Slota update); ~0 before
};

// A control block reset on the device (k_canon_write), as the host would
// initialise it: zero, then the fields below; pivkey: one pivot word to
// clear as well, or nullptr.
struct CtlReset {
    Ctl *next;
    unsigned long long timeout_ns;
    unsigned long long *trace;
    unsigned trace_cap;
    unsigned long long *pivkey;
};

// Phase ids recorded in the pass trace.
enum {
    PH_INIT = 1, PH_TRIM1_ONCE = 2, PH_TRIM1_APPLY = 3, PH_TRIM1_FIX = 4, PH_TRIM2 = 5, PH_TRIM2_APPLY = 6,
    PH_FIRST_PIVOT = 7, PH_BFS0 = 8, PH_BFS = 9, PH_PROP = 10, PH_HONG_UPDATE = 11, PH_SLOTA_FIRST_UPDATE = 12,
    PH_SLOTA_PEEL_UPDATE = 13, PH_RENAME = 14, PH_PIVOTS = 15, PH_BFS_PULL = 16, PH_PROP_PULL = 17,
    PH_RES_TAG = 18, PH_RES_EXTRACT = 19, PH_RES_SOLVE = 20
};

struct Graph {
    uint32_t V, E;
    const uint32_t *__restrict__ Fr, *__restrict__ Fc, *__restrict__ Br, *__restrict__ Bc;
    uint32_t vec;   // Fr and Br are 16-byte aligned: 128-bit offset loads allowed
};

// o[0..4] = R[i0 .. i0+4] with indices clipped to V+1 (the last offset);
// one 128-bit load plus one 32-bit load when R is 16-byte aligned (i0 is a
// multiple of 4).
__device__ __forceinline__ void load_off5(const uint32_t *__restrict__ R, uint32_t i0, uint32_t V, uint32_t vec,
                                          uint32_t (&o)[5])
{
    if (vec && i0 + 4u <= V + 1u) {
        const uint4 x = __ldg(reinterpret_cast<const uint4 *>(R + i0));
        o[0] = x.x; o[1] = x.y; o[2] = x.z; o[3] = x.w;
        o[4] = __ldg(&R[i0 + 4u]);
    } else {
#pragma unroll
        for (int j = 0; j < 5; j++) o[j] = __ldg(&R[min(i0 + (uint32_t)j, V + 1u)]);
    }
}

struct Work {
    uint32_t *st, *label, *stamp;
    uint32_t *smin;             // smin[r] = smallest member id of the SCC represented by r; set to r
                                // when r becomes a representative (its seed pass), then folded
    uint32_t *L[2];
    uint32_t *S[2];             // whole-GPU path: lists of the shrinking bottom-up scope (nullptr elsewhere)
    uint32_t *Q[2][2];          // [direction][parity]
    uint2 *H[2][2];             // heavy chunks (vertex, chunk) [direction][parity]
    uint32_t hcap;
    unsigned long long *pivkey; // Hong: 4V+4 slots; Slota: 1
    Ctl *ctl;
    uint32_t qcap;              // entries per CTA staging queue (dynamic shared memory)
    uint32_t bu_k;              // bottom-up BFS step when frontier edges > bu_k * scope vertices (0 = never)
    uint32_t pull_lane;         // bottom-up step: lists up to this many entries are tested by their lane alone;
                                // of a longer list the lane tests the first min(8, pull_lane), the warp the rest
};

constexpr uint32_t PULL_LANE = 32;   // Work::pull_lane of the batched and no-allocation paths

// Carve the work arrays for a graph of V vertices and E edges out of `base`
// (nullptr: only count).  Returns the bytes used.  Same layout on host and
// device; used by the batched form, where every CTA re-carves its private
// scratch for each graph it takes.
__host__ __device__ inline size_t carve_work(char *base, uint32_t V, uint32_t E, bool hong, Work *w)
{
    const size_t n1 = (size_t)V + 1;
    const size_t hcap = (size_t)E / CH + (size_t)E / HEAVY_T + 64;
    const size_t va = (n1 * 4 + 255) / 256 * 256;       // one vertex array
    const size_t ha = (hcap * 8 + 255) / 256 * 256;     // one chunk queue
    const size_t pa = ((hong ? 4 * n1 + 8 : 1) * 8 + 255) / 256 * 256;
    const size_t ca = (sizeof(Ctl) + 255) / 256 * 256;
    if (w && base) {
        w->st = (uint32_t *)(base);
        w->label = (uint32_t *)(base + va);
        w->stamp = (uint32_t *)(base + 2 * va);
        w->smin = (uint32_t *)(base + 3 * va);
        w->L[0] = (uint32_t *)(base + 4 * va);
        w->L[1] = (uint32_t *)(base + 5 * va);
        w->S[0] = w->S[1] = nullptr;
        w->Q[0][0] = (uint32_t *)(base + 6 * va);
        w->Q[0][1] = (uint32_t *)(base + 7 * va);
        w->Q[1][0] = (uint32_t *)(base + 8 * va);
        w->Q[1][1] = (uint32_t *)(base + 9 * va);
        w->H[0][0] = (uint2 *)(base + 10 * va);
        w->H[0][1] = (uint2 *)(base + 10 * va + ha);
        w->H[1][0] = (uint2 *)(base + 10 * va + 2 * ha);
        w->H[1][1] = (uint2 *)(base + 10 * va + 3 * ha);
        w->hcap = (uint32_t)hcap;
        w->pivkey = (unsigned long long *)(base + 10 * va + 4 * ha);
        w->ctl = (Ctl *)(base + 10 * va + 4 * ha + pa);
    }
    return 10 * va + 4 * ha + pa + ca;
}

// Dynamic shared memory of the SCC kernels: BQ_HDR control words, then the
// staging queues (at most NBQ: two frontier queues, and on the whole-GPU
// kernel a third one for the shrinking bottom-up scope), each split into
// one slice of qcap entries per warp of the CTA: (BQ_HDR + queues * warps *
// qcap) words.
constexpr unsigned NBQ = 3;
constexpr unsigned BQ_WARPS = 32;                       // at most 1024 threads per CTA
constexpr unsigned BQ_CNT = 16;                         // per-warp fill counts [NBQ][BQ_WARPS]
constexpr unsigned BQ_PRE = BQ_CNT + NBQ * BQ_WARPS;    // per-warp flush offsets [NBQ][BQ_WARPS]
constexpr unsigned BQ_HDR = BQ_PRE + NBQ * BQ_WARPS;
extern __shared__ uint32_t sccb_dsmem[];

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned vld(const unsigned *p) { return *(const volatile unsigned *)p; }
// The CTA's own copy of "an error was set", read by the single-CTA
// barrier instead of the control block's word (one load from L2 less per
// pass); every set_error raises it.
__device__ __forceinline__ int *cta_err()
{
    __shared__ int s_cta_err;
    return &s_cta_err;
}

__device__ __forceinline__ void set_error(Ctl *c, int code, int where)
{
    *(volatile int *)cta_err() = 1;
    if (atomicCAS(&c->error, 0, code) == 0) c->where = where;
}

// Adjacency ids must lie in [1, V].  An id outside that range is reported
// as a malformed graph and treated as vertex 0, which is permanently dead,
// so no state array is ever indexed out of bounds.
__device__ __forceinline__ uint32_t guard_id(uint32_t x, uint32_t V, Ctl *c)
{
    if (x - 1u >= V) {
        set_error(c, E_BAD_GRAPH, 60);
        return 0u;
    }
    return x;
}

// ---------------------------------------------------------------------
// execution policies
// ---------------------------------------------------------------------
// Per-CTA copy of the counters the last pass pushed (written by thread 0
// right after the pass barrier, read by every thread through last_count):
// one load per CTA instead of one per warp on the same few words, which made
// a same-address hot spot in L2 on every pass.
__device__ __forceinline__ unsigned *cnt_snap()
{
    __shared__ unsigned s_cnt[NCNT];
    return s_cnt;
}
// Pass counter ring of the single-CTA policy (BlockExec): in shared memory,
// since no other CTA reads it.
__device__ __forceinline__ unsigned (*block_lc())[NCNT]
{
    __shared__ unsigned s_lc[3][NCNT];
    return s_lc;
}

__device__ __forceinline__ void take_snap(const unsigned *c)
{
    unsigned *d = cnt_snap();
#pragma unroll
    for (int i = 0; i < NCNT; i++) d[i] = *(volatile const unsigned *)&c[i];
}

template <bool INSTR>
struct GridExec {
    static constexpr bool instr = INSTR;
    static constexpr bool grid = true;
    static constexpr bool cluster = false;
    static constexpr unsigned nbq = 3;   // staging queues of the launch's shared memory
    Ctl *ctl;
    unsigned gl;        // pass counter, identical in every thread
    unsigned cap = 0;   // pass cap of the run (0: none), see run_pass
    unsigned hold = 0;  // failure-detection test hook, see sync
    __device__ __forceinline__ unsigned tid() const { return blockIdx.x * blockDim.x + threadIdx.x; }
    __device__ __forceinline__ unsigned nthr() const { return gridDim.x * blockDim.x; }
    __device__ __forceinline__ unsigned wid() const { return tid() >> 5; }
    __device__ __forceinline__ unsigned nwarps() const { return nthr() >> 5; }
    __device__ __forceinline__ bool leader() const { return blockIdx.x == 0 && threadIdx.x == 0; }
    __device__ __forceinline__ unsigned *lc(unsigned slot) const { return ctl->lc[slot]; }

    // Grid barrier.  One arrival counter: CTA 0 adds 0x80000000 - (n - 1),
    // every other CTA adds 1, so bit 31 flips exactly when all n CTAs have
    // arrived.  Arrival is a release, the flip is read with acquire.  A
    // waiter leaves early when the sticky error word (polled with the
    // counter in one 8-byte load) is set, or after ctl->timeout_ns; any CTA
    // that sees an error returns, and the error stays set for the others.
    //
    // hold = k + 1 makes the last CTA withhold its arrival at pass k: the
    // failure-detection tests use it to make every wait of that barrier run
    // out (an arrival that never comes), which must end the run with
    // E_TIMEOUT and leave the context usable.
    __device__ bool sync(const unsigned *snap = nullptr)
    {
        __shared__ int s_err;
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned nb = (blockIdx.x == 0) ? (0x80000000u - (gridDim.x - 1u)) : 1u;
            unsigned old;
            if (hold != 0u && gl + 1u == hold && blockIdx.x == gridDim.x - 1u)
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(old) : "l"(&ctl->bar_count) : "memory");
            else
                asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(&ctl->bar_count), "r"(nb) : "memory");
            int err = 0;
            unsigned long long t0 = 0;
            for (unsigned spin = 0;; spin++) {
                unsigned long long wv;
                asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(wv) : "l"(&ctl->bar_count) : "memory");
                err = (int)(wv >> 32);
                if ((((unsigned)wv ^ old) & 0x80000000u) != 0u || err) break;
                if ((spin & 255u) == 0u) {
                    unsigned long long t = gtimer();
                    if (spin == 0) t0 = t;
                    else if (t - t0 > ctl->timeout_ns) {
                        set_error(ctl, E_TIMEOUT, 1000);
                        err = E_TIMEOUT;
                        break;
                    }
                }
            }
            s_err = err;
            if (snap) take_snap(snap);
        }
        __syncthreads();
        return s_err == 0;
    }
};

template <bool INSTR>
struct BlockExec {
    static constexpr bool instr = INSTR;
    static constexpr bool grid = false;
    static constexpr bool cluster = false;
    static constexpr unsigned nbq = 2;
    Ctl *ctl;
    unsigned gl;
    unsigned cap = 0;
    __device__ __forceinline__ unsigned tid() const { return threadIdx.x; }
    __device__ __forceinline__ unsigned nthr() const { return blockDim.x; }
    __device__ __forceinline__ unsigned wid() const { return threadIdx.x >> 5; }
    __device__ __forceinline__ unsigned nwarps() const { return blockDim.x >> 5; }
    __device__ __forceinline__ bool leader() const { return threadIdx.x == 0; }
    __device__ __forceinline__ unsigned *lc(unsigned slot) const { return block_lc()[slot]; }
    // Counters and the error flag of a new run on this CTA (every thread calls).
    __device__ void reset_counters() const
    {
        for (unsigned i = threadIdx.x; i < 3u * NCNT; i += blockDim.x) (&block_lc()[0][0])[i] = 0u;
        if (threadIdx.x == 0) *cta_err() = *(volatile int *)&ctl->error != 0;
        __syncthreads();
    }
    __device__ bool sync(const unsigned *snap = nullptr)
    {
        __shared__ int s_err;
        __syncthreads();
        if (threadIdx.x == 0) {
            s_err = *(volatile int *)cta_err();
            if (snap) take_snap(snap);
        }
        __syncthreads();
        return s_err == 0;
    }
};

__device__ __forceinline__ unsigned cluster_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_size()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
// Hardware cluster barrier (every thread of every CTA of the cluster);
// writes before it, in any state space, are visible to the whole cluster
// after it.
__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// One graph on the CTAs of a thread-block cluster (co-scheduled by the
// hardware, so the barrier is the cluster barrier and needs no timeout).
// The error word is read between two barriers: no pass body runs while
// any CTA reads it, so every CTA takes the same branch.
//
// With `soft` set, the barrier is instead a counter in global memory (the
// grid barrier's bit-flip scheme over the cluster's CTAs) whose waits give
// up after soft_timeout_ns with E_TIMEOUT: a check mode in which a
// mismatch of barrier counts between the CTAs ends in an error status
// rather than a wait that never ends.
template <bool INSTR>
struct ClusterExec {
    static constexpr bool instr = INSTR;
    static constexpr bool grid = false;
    static constexpr bool cluster = true;
    static constexpr unsigned nbq = 2;
    Ctl *ctl;
    unsigned gl;
    unsigned rank, csize;
    unsigned *soft;   // the cluster's barrier counter, or nullptr for the hardware barrier
    unsigned long long soft_timeout_ns;
    unsigned cap = 0;
    unsigned hold = 0;  // check mode only: the last CTA withholds its arrival at pass hold - 1 (test hook)
    __device__ __forceinline__ unsigned tid() const { return rank * blockDim.x + threadIdx.x; }
    __device__ __forceinline__ unsigned nthr() const { return csize * blockDim.x; }
    __device__ __forceinline__ unsigned wid() const { return tid() >> 5; }
    __device__ __forceinline__ unsigned nwarps() const { return nthr() >> 5; }
    __device__ __forceinline__ bool leader() const { return rank == 0 && threadIdx.x == 0; }
    __device__ __forceinline__ unsigned *lc(unsigned slot) const { return ctl->lc[slot]; }
    __device__ void barrier()
    {
        if (!soft) {
            cluster_barrier();
            return;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned nb = rank == 0 ? (0x80000000u - (csize - 1u)) : 1u;
            unsigned old;
            if (hold != 0u && gl + 1u == hold && rank == csize - 1u)
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(old) : "l"(soft) : "memory");
            else
                asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(soft), "r"(nb) : "memory");
            unsigned long long t0 = 0;
            for (unsigned spin = 0;; spin++) {
                unsigned v;
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(soft) : "memory");
                if (((v ^ old) & 0x80000000u) != 0u) break;
                if ((spin & 255u) == 0u) {
                    const unsigned long long t = gtimer();
                    if (spin == 0) t0 = t;
                    else if (t - t0 > soft_timeout_ns) {
                        set_error(ctl, E_TIMEOUT, 1001);
                        break;
                    }
                }
            }
        }
        __syncthreads();
    }
    __device__ bool sync(const unsigned *snap = nullptr)
    {
        __shared__ int s_err;
        barrier();
        if (threadIdx.x == 0) {
            s_err = *(volatile int *)&ctl->error;
            if (snap) take_snap(snap);
        }
        barrier();
        return s_err == 0;
    }
};

// One pass: clear the counters the pass after next will push into, run the
// body with (cur, nxt) counter slots, then the barrier.  A pass pushes into
// counter slot gl%3 and buffer parity gl&1; the following pass reads them as
// its "current" slot (gl+2)%3 and parity (gl+1)&1.
//
// A run whose pass count reaches ex.cap (when set) stops with
// E_NOT_CONVERGED: the host's bound on the work of one run, on top of the
// V + 2 passes every convergence loop allows itself.
template <class Ex, class F>
__device__ __forceinline__ bool run_pass(Ex &ex, int phase, F &&body)
{
    if (ex.cap != 0u && ex.gl >= ex.cap) {
        if (ex.leader()) set_error(ex.ctl, E_NOT_CONVERGED, 70);
        ex.sync();
        ex.gl++;
        return false;
    }
    const unsigned nxt = ex.gl % 3u, clr = (ex.gl + 1u) % 3u, cur = (ex.gl + 2u) % 3u;
    if (ex.leader()) {
#pragma unroll
        for (int i = 0; i < NCNT; i++) ex.lc(clr)[i] = 0u;
    }
    body(cur, nxt);
    bool ok = ex.sync(ex.lc(nxt));
    if (ex.leader() && ex.ctl->trace && ex.gl < ex.ctl->trace_cap) {
        // pass trace: end time and (phase, items pushed) -- the reference's
        // _DEBUG per-phase event timers (scc_WCC.cu:650-672) at pass granularity
        // (instrumented runs record the running count of adjacency entries scanned instead)
        const unsigned *c = ex.lc(nxt);
        unsigned long long pushed = (unsigned long long)vld(&c[C_FQ]) + vld(&c[C_BQ]) + vld(&c[C_LIST]);
        if constexpr (Ex::instr) pushed = *(volatile unsigned long long *)&ex.ctl->t_edges;
        ex.ctl->trace[2 * ex.gl] = gtimer();
        ex.ctl->trace[2 * ex.gl + 1] = (unsigned long long)phase | (pushed << 8);
    }
    ex.gl++;
    return ok;
}

// Counter value pushed by the pass that just finished (the CTA's snapshot).
template <class Ex>
__device__ __forceinline__ unsigned last_count(const Ex &, int which)
{
    return cnt_snap()[which];
}

// ---------------------------------------------------------------------
// warp primitives
// ---------------------------------------------------------------------

// Warp-aggregated append (ballot + one atomicAdd per warp): the frontier
// compaction.  All 32 lanes must call it.
__device__ __forceinline__ void warp_push(bool pred, uint32_t val, uint32_t *q, unsigned *cnt,
                                          uint32_t cap, Ctl *ctl, int where)
{
    unsigned m = __ballot_sync(FULL, pred);
    if (m == 0u) return;
    unsigned lane = lane_id();
    unsigned ld = __ffs(m) - 1u;
    unsigned base = 0;
    if (lane == ld) base = atomicAdd(cnt, (unsigned)__popc(m));
    base = __shfl_sync(FULL, base, ld);
    if (pred) {
        unsigned pos = base + __popc(m & ((1u << lane) - 1u));
        if (pos < cap) q[pos] = val;
        else set_error(ctl, E_OVERFLOW, where);
    }
}

// Staging of queue appends in shared memory: every warp appends into its
// own slice (warp ballot, no atomics); a full slice is written out by its
// warp with one global atomicAdd per qcap entries, and bq_flush writes the
// rest of all slices with one global atomicAdd per CTA and pass.  This keeps
// the global queue tail from becoming a same-address atomic hot spot.
__device__ __forceinline__ uint32_t *cta_first_min();
__device__ __forceinline__ void bq_init()
{
    for (unsigned i = threadIdx.x; i < BQ_HDR; i += blockDim.x) sccb_dsmem[i] = 0u;
    if (threadIdx.x == 0) {
        *cta_first_min() = 0xFFFFFFFFu;
        *cta_err() = 0;
    }
    __syncthreads();
}

__device__ __forceinline__ void bq_push(unsigned qi, bool pred, uint32_t val, uint32_t qcap, uint32_t *gq,
                                        unsigned *gcnt, uint32_t gcap, Ctl *ctl, int where)
{
    const unsigned m = __ballot_sync(FULL, pred);
    if (m == 0u) return;
    const unsigned lane = lane_id(), wi = threadIdx.x >> 5;
    uint32_t *slice = &sccb_dsmem[BQ_HDR + (qi * (blockDim.x >> 5) + wi) * qcap];
    unsigned *wc = &sccb_dsmem[BQ_CNT + qi * BQ_WARPS + wi];
    unsigned cnt = *wc;
    const unsigned n = __popc(m);
    if (cnt + n > qcap) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(gcnt, cnt);
        base = __shfl_sync(FULL, base, 0);
        for (unsigned i = lane; i < cnt; i += 32u) {
            if (base + i < gcap) gq[base + i] = slice[i];
            else set_error(ctl, E_OVERFLOW, where);
        }
        __syncwarp();
        cnt = 0;
    }
    if (pred) slice[cnt + __popc(m & ((1u << lane) - 1u))] = val;
    __syncwarp();
    if (lane == 0) *wc = cnt + n;
    __syncwarp();
}

// Adds x to the CTA's frontier-edge tally of queue qi (words 12, 13).
__device__ __forceinline__ void bq_add_edges(unsigned qi, unsigned x)
{
    x = __reduce_add_sync(FULL, x);
    if (lane_id() == 0 && x) atomicAdd(&sccb_dsmem[12 + qi], x);
}

// Called by every thread of the CTA at the end of a pass.  ecnt0 / ecnt1
// (optional) receive the CTA's frontier-edge tallies.
__device__ __forceinline__ void bq_flush(unsigned nq, uint32_t qcap, uint32_t *gq0, unsigned *gcnt0, uint32_t *gq1,
                                         unsigned *gcnt1, uint32_t gcap, Ctl *ctl, unsigned *ecnt0 = nullptr,
                                         unsigned *ecnt1 = nullptr, uint32_t *gq2 = nullptr, unsigned *gcnt2 = nullptr)
{
    __syncthreads();
    const unsigned nw = blockDim.x >> 5;
    const unsigned wi = threadIdx.x >> 5;
    // warp q lays out queue q: the warps' fill counts scanned by shuffles,
    // one global atomicAdd for the CTA's room; the queues' atomics overlap
    for (unsigned qi = wi; qi < nq; qi += nw) {
        const unsigned ln = lane_id();
        const unsigned c = ln < nw ? sccb_dsmem[BQ_CNT + qi * BQ_WARPS + ln] : 0u;
        unsigned incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(FULL, incl, o);
            if (ln >= (unsigned)o) incl += y;
        }
        if (ln < nw) sccb_dsmem[BQ_PRE + qi * BQ_WARPS + ln] = incl - c;
        const unsigned total = __shfl_sync(FULL, incl, 31);
        if (ln == 0) {
            sccb_dsmem[8 + qi] = total ? atomicAdd(qi == 2 ? gcnt2 : qi ? gcnt1 : gcnt0, total) : 0u;
            unsigned *ec = qi == 2 ? nullptr : qi ? ecnt1 : ecnt0;
            if (ec && sccb_dsmem[12 + qi]) atomicAdd(ec, sccb_dsmem[12 + qi]);
            sccb_dsmem[12 + qi] = 0u;
        }
    }
    __syncthreads();
    for (unsigned qi = 0; qi < nq; qi++) {
        uint32_t *gq = qi == 2 ? gq2 : qi ? gq1 : gq0;
        const unsigned cnt = sccb_dsmem[BQ_CNT + qi * BQ_WARPS + wi];
        const unsigned base = sccb_dsmem[8 + qi] + sccb_dsmem[BQ_PRE + qi * BQ_WARPS + wi];
        const uint32_t *slice = &sccb_dsmem[BQ_HDR + (qi * nw + wi) * qcap];
        for (unsigned i = lane_id(); i < cnt; i += 32u) {
            if (base + i < gcap) gq[base + i] = slice[i];
            else set_error(ctl, E_OVERFLOW, 3);
        }
        __syncwarp();
        if (lane_id() == 0) sccb_dsmem[BQ_CNT + qi * BQ_WARPS + wi] = 0u;
    }
}

// Per-CTA minimum of the vertices whose second visited bit (FV then BV or
// BV then FV) was set by this CTA: the members of the first pivot's SCC
// during the first search.  Cleared at kernel entry (bq_init).
__device__ __forceinline__ uint32_t *cta_first_min()
{
    __shared__ uint32_t s_first_min;
    return &s_first_min;
}
// old: the state word before an atomicOr of `bits`: v if that atomicOr
// completed both visited bits, else ~0.
__device__ __forceinline__ uint32_t completed(uint32_t old, uint32_t bits, uint32_t v)
{
    return ((old & (FVB | BVB)) != (FVB | BVB) && ((old | bits) & (FVB | BVB)) == (FVB | BVB)) ? v : 0xFFFFFFFFu;
}
// Folds the warp's smallest completed vertex into the CTA's minimum: one
// warp reduction, and a shared-memory atomic only when it lowers the CTA's
// current value (the first SCC's smallest member is found early, so almost
// every call ends at the comparison).  All 32 lanes call.
__device__ __forceinline__ void fold_completed(uint32_t cand)
{
    const uint32_t m = __reduce_min_sync(0xFFFFFFFFu, cand);
    if ((threadIdx.x & 31u) == 0u && m < *(volatile uint32_t *)cta_first_min()) atomicMin(cta_first_min(), m);
}

// Adds the CTA's frontier-edge tally of queue 0 (word 12) to *ecnt and
// clears it: the end of a pass that tallies without staging queues.
// Called by every thread of the CTA.
__device__ __forceinline__ void bq_flush_edges(unsigned *ecnt)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        if (sccb_dsmem[12]) atomicAdd(ecnt, sccb_dsmem[12]);
        sccb_dsmem[12] = 0u;
    }
}

__device__ __forceinline__ unsigned warp_incl_scan(unsigned x)
{
    unsigned lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(FULL, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    return x;
}

// Append nch chunk descriptors (v, 0..nch-1) per lane.  All lanes call.
__device__ __forceinline__ void warp_push_chunks(uint32_t v, uint32_t nch, uint2 *hq, unsigned *hcnt,
                                                 uint32_t hcap, Ctl *ctl)
{
    unsigned incl = warp_incl_scan(nch);
    unsigned total = __shfl_sync(FULL, incl, 31);
    if (total == 0u) return;
    unsigned base = 0;
    if (lane_id() == 0) base = atomicAdd(hcnt, total);
    base = __shfl_sync(FULL, base, 0);
    unsigned pos = base + incl - nch;
    if (pos + nch > hcap) { if (nch) set_error(ctl, E_OVERFLOW, 2); return; }
    for (uint32_t c = 0; c < nch; c++) hq[pos + c] = make_uint2(v, c);
}

// First pusher of u for pass tag wins (stamp dedup of work lists).
__device__ __forceinline__ bool stamp_claim(uint32_t *stamp, uint32_t u, uint32_t tag)
{
    if (stamp[u] >= tag) return false;
    return atomicMax(&stamp[u], tag) < tag;
}

// Load-balanced expansion of up to 32 adjacency lists held one per lane
// (merge-path style): the warp walks the concatenation of the lists 32
// entries at a time, each lane finds its owner by a 5-step binary search
// over the exclusive scan of the degrees.  fn(valid, neighbour, aux_of_owner)
// is called by all lanes on every step.  Degrees must be <= HEAVY_T.
template <class Fn>
__device__ __forceinline__ unsigned lbs_expand(uint32_t beg, uint32_t deg, uint32_t aux,
                                               const uint32_t *__restrict__ C, Fn &&fn)
{
    unsigned incl = warp_incl_scan(deg);
    unsigned total = __shfl_sync(FULL, incl, 31);
    unsigned excl = incl - deg;
    unsigned lane = lane_id();
    for (unsigned base = 0; base < total; base += 32u) {
        unsigned e = base + lane;
        unsigned lo = 0;
#pragma unroll
        for (unsigned step = 16; step >= 1; step >>= 1) {
            unsigned cand = lo + step;
            unsigned x = __shfl_sync(FULL, excl, cand & 31u);
            if (cand < 32u && x <= e) lo = cand;
        }
        unsigned ex_o = __shfl_sync(FULL, excl, lo);
        unsigned beg_o = __shfl_sync(FULL, beg, lo);
        unsigned aux_o = __shfl_sync(FULL, aux, lo);
        bool valid = e < total;
        uint32_t nbr = valid ? __ldg(&C[beg_o + (e - ex_o)]) : 0u;
        fn(valid, nbr, aux_o);
    }
    return total;
}

// Same walk, two entries per lane per step so that each lane has two
// independent gathers in flight: fn(v0, n0, aux0, v1, n1, aux1).
template <class Fn>
__device__ __forceinline__ unsigned lbs_expand2(uint32_t beg, uint32_t deg, uint32_t aux,
                                                const uint32_t *__restrict__ C, Fn &&fn)
{
    unsigned incl = warp_incl_scan(deg);
    unsigned total = __shfl_sync(FULL, incl, 31);
    unsigned excl = incl - deg;
    unsigned lane = lane_id();
    for (unsigned base = 0; base < total; base += 64u) {
        const unsigned e0 = base + lane, e1 = e0 + 32u;
        unsigned lo0 = 0, lo1 = 0;
#pragma unroll
        for (unsigned step = 16; step >= 1; step >>= 1) {
            unsigned c0 = lo0 + step, c1 = lo1 + step;
            unsigned x0 = __shfl_sync(FULL, excl, c0 & 31u);
            unsigned x1 = __shfl_sync(FULL, excl, c1 & 31u);
            if (c0 < 32u && x0 <= e0) lo0 = c0;
            if (c1 < 32u && x1 <= e1) lo1 = c1;
        }
        const unsigned x0 = __shfl_sync(FULL, excl, lo0), x1 = __shfl_sync(FULL, excl, lo1);
        const unsigned b0 = __shfl_sync(FULL, beg, lo0), b1 = __shfl_sync(FULL, beg, lo1);
        const unsigned a0 = __shfl_sync(FULL, aux, lo0), a1 = __shfl_sync(FULL, aux, lo1);
        const bool v0 = e0 < total, v1 = e1 < total;
        const uint32_t n0 = v0 ? __ldg(&C[b0 + (e0 - x0)]) : 0u;
        const uint32_t n1 = v1 ? __ldg(&C[b1 + (e1 - x1)]) : 0u;
        fn(v0, n0, a0, v1, n1, a1);
    }
    return total;
}

// Fold member v into smin[rep] (the canonical label of rep's SCC): lanes
// sharing rep reduce first, one atomicMin per group, skipped when the
// stored value is already smaller.  All 32 lanes call.
__device__ __forceinline__ void smin_fold(bool valid, uint32_t rep, uint32_t v, uint32_t *smin)
{
    const unsigned vm = __ballot_sync(FULL, valid);
    if (vm == 0u) return;
    const uint32_t rep0 = __shfl_sync(FULL, rep, __ffs(vm) - 1);
    if (__all_sync(FULL, !valid || rep == rep0)) {   // one SCC for the whole warp (the common case)
        const uint32_t mn = __reduce_min_sync(FULL, valid ? v : 0xFFFFFFFFu);
        if (lane_id() == 0 && mn < vld(&smin[rep0])) atomicMin(&smin[rep0], mn);
        return;
    }
    unsigned grp = __match_any_sync(FULL, valid ? rep : 0xFFFFFFFFu);
    uint32_t mn = __reduce_min_sync(grp, valid ? v : 0xFFFFFFFFu);
    if (valid && lane_id() == (unsigned)(__ffs(grp) - 1) && mn < vld(&smin[rep])) atomicMin(&smin[rep], mn);
}

// Virtual-warp expansion: groups of W = 1 << lw lanes share one vertex and
// stride over its adjacency (the reference's fwd_warp/bwd_warp schedule,
// include/scc_kernels.h:46-105).  Returns the entries scanned by the warp.
template <class Fn>
__device__ __forceinline__ unsigned vw_expand(uint32_t beg, uint32_t deg, uint32_t aux, unsigned lw,
                                              const uint32_t *__restrict__ C, Fn &&fn)
{
    unsigned W = 1u << lw;
    unsigned sub = lane_id() & (W - 1u);
    unsigned maxd = __reduce_max_sync(FULL, deg);
    for (unsigned base = 0; base < maxd; base += W) {
        unsigned k = base + sub;
        bool valid = k < deg;
        uint32_t nbr = valid ? __ldg(&C[beg + k]) : 0u;
        fn(valid, nbr, aux);
    }
    unsigned own = (sub == 0u) ? deg : 0u;
    return __reduce_add_sync(FULL, own);
}

// Virtual-warp expansion of K vertices per lane group at once (the same W
// lanes per vertex as vw_expand): the K lists are walked in the same steps,
// so every lane has K gathers in flight.  fn(j, valid, nbr) per entry, in
// pairs of j; returns the entries of the warp.
template <int K, class Fn>
__device__ __forceinline__ unsigned vw_expandK(const uint32_t (&beg)[K], const uint32_t (&deg)[K], unsigned lw,
                                               const uint32_t *__restrict__ C, Fn &&fn)
{
    const unsigned W = 1u << lw;
    const unsigned sub = lane_id() & (W - 1u);
    unsigned md = 0, own = 0;
#pragma unroll
    for (int j = 0; j < K; j++) {
        md = max(md, deg[j]);
        own += deg[j];
    }
    const unsigned maxd = __reduce_max_sync(FULL, md);
    for (unsigned base = 0; base < maxd; base += W) {
        const unsigned k = base + sub;
        uint32_t n[K];
        bool v[K];
#pragma unroll
        for (int j = 0; j < K; j++) {
            v[j] = k < deg[j];
            n[j] = v[j] ? __ldg(&C[beg[j] + k]) : 0u;
        }
#pragma unroll
        for (int j = 0; j < K; j += 2) fn(j, v[j], n[j], v[j + 1], n[j + 1]);
    }
    return __reduce_add_sync(FULL, sub == 0u ? own : 0u);
}

// Minimum of x over the CTA folded into *dst with one atomicMin by thread 0
// (skipped when *dst is already smaller).  Called by every thread of the
// CTA; 0xFFFFFFFF means "nothing".  Used where every member found in a pass
// belongs to the same SCC, so its canonical label needs one atomic per CTA
// rather than one per warp on the same word.
__device__ __forceinline__ void block_min_atomic(uint32_t x, uint32_t *dst)
{
    __shared__ uint32_t s_min[32];
    const uint32_t m = __reduce_min_sync(FULL, x);
    const unsigned wi = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane_id() == 0) s_min[wi] = m;
    __syncthreads();
    if (wi == 0) {
        const uint32_t r = __reduce_min_sync(FULL, lane_id() < nw ? s_min[lane_id()] : 0xFFFFFFFFu);
        if (lane_id() == 0 && r != 0xFFFFFFFFu && r < *(volatile uint32_t *)dst) atomicMin(dst, r);
    }
    __syncthreads();
}

// 32-bit max over the warp, then the CTA; the CTA's thread 0 performs one
// atomicMax.  Called by every thread of the CTA.
__device__ __forceinline__ void block_max_atomic32(uint32_t x, uint32_t *dst)
{
    __shared__ uint32_t s_max[32];
    const uint32_t m = __reduce_max_sync(FULL, x);
    const unsigned wi = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane_id() == 0) s_max[wi] = m;
    __syncthreads();
    if (wi == 0) {
        const uint32_t r = __reduce_max_sync(FULL, lane_id() < nw ? s_max[lane_id()] : 0u);
        if (lane_id() == 0 && r > *(volatile uint32_t *)dst) atomicMax(dst, r);
    }
    __syncthreads();
}

// 64-bit max of a pivot key over the warp, then the CTA; the CTA's thread 0
// performs one atomicMax.  With dst32 set, the 32-bit max of x goes to
// dst32 in the same two barriers.  Called by every thread of the CTA.
__device__ __forceinline__ void block_max_atomic(unsigned long long key, unsigned long long *dst, uint32_t x = 0u,
                                                 uint32_t *dst32 = nullptr)
{
    __shared__ unsigned long long s_red[32];
    __shared__ uint32_t s_x[32];
    unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
    unsigned mhi = __reduce_max_sync(FULL, hi);
    unsigned mlo = __reduce_max_sync(FULL, hi == mhi ? lo : 0u);
    unsigned long long wk = ((unsigned long long)mhi << 32) | mlo;
    unsigned w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t mx = dst32 ? __reduce_max_sync(FULL, x) : 0u;
    if (lane_id() == 0) { s_red[w] = wk; s_x[w] = mx; }
    __syncthreads();
    if (w == 0) {
        const unsigned long long k = lane_id() < nw ? s_red[lane_id()] : 0ull;
        const unsigned khi = __reduce_max_sync(FULL, (unsigned)(k >> 32));
        const unsigned klo = __reduce_max_sync(FULL, (unsigned)(k >> 32) == khi ? (unsigned)k : 0u);
        const unsigned long long m = ((unsigned long long)khi << 32) | klo;
        if (lane_id() == 0 && m && m > *(volatile unsigned long long *)dst) atomicMax(dst, m);
        if (dst32) {
            const uint32_t r = __reduce_max_sync(FULL, lane_id() < nw ? s_x[lane_id()] : 0u);
            if (lane_id() == 0 && r > *(volatile uint32_t *)dst32) atomicMax(dst32, r);
        }
    }
    __syncthreads();
}

// Pivot key (scc_kernels.cu:643-656): uint32 product of full-graph out- and
// in-degree, larger wins; ties go to the smaller id.  Never 0 for v <= MAX_V.
__device__ __forceinline__ unsigned long long pivot_key(const Graph &g, uint32_t v)
{
    uint32_t prod = (__ldg(&g.Fr[v + 1]) - __ldg(&g.Fr[v])) * (__ldg(&g.Br[v + 1]) - __ldg(&g.Br[v]));
    return ((unsigned long long)prod << 32) | (unsigned long long)(0xFFFFFFFFu - v);
}
__device__ __forceinline__ uint32_t key_vertex(unsigned long long k) { return 0xFFFFFFFFu - (uint32_t)k; }

// Range names after a FW-BW split: three fresh names per pivot.  The
// reference uses 3*range + FV + 2*BV (scc_kernels.cu:138), which wraps.
__device__ __forceinline__ uint32_t split_name(uint32_t V, uint32_t p, uint32_t s)
{
    return (V + 1u) + 3u * p + ((s & FVB) ? 1u : 0u) + ((s & BVB) ? 2u : 0u);
}

// Per-range atomicMax of pivot keys with warp aggregation over lanes that
// share a range (match.any + redux) and a read before the atomic.
// Returns true in exactly one lane of the whole launch per range: the one
// whose atomicMax found the slot still empty (the range's first bid).
__device__ __forceinline__ bool range_max_atomic(bool valid, uint32_t r, unsigned long long key,
                                                 unsigned long long *pivkey)
{
    unsigned grp = __match_any_sync(FULL, valid ? r : 0xFFFFFFFFu);
    unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
    unsigned mhi = __reduce_max_sync(grp, hi);
    unsigned mlo = __reduce_max_sync(grp, hi == mhi ? lo : 0u);
    bool first = false;
    if (valid && lane_id() == (unsigned)(__ffs(grp) - 1)) {
        unsigned long long k = ((unsigned long long)mhi << 32) | mlo;
        if (k > *(volatile unsigned long long *)&pivkey[r]) first = atomicMax(&pivkey[r], k) == 0ull;
    }
    return first;
}

}  // namespace sccb
