// Kernels and host side of the C ABI (include/scc_b200.h).
//
// One scc_run = (optional H2D copies) -> one SCC launch (cooperative
// whole-GPU persistent kernel, or one CTA for small graphs; its first pass
// also validates the offsets) -> one canonical-label kernel -> (optional D2H
// of labels) -> one D2H of the control block.  The reference instead issues one launch plus
// one or two blocking 1-byte copies per BFS level and per propagation sweep
// (e.g. scc_WCC.cu:880-885).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>

#include "../../include/scc_b200.h"
#include "scc_phases.cuh"
#include "scc_internal.h"

using namespace sccb;

#define SCC_VERSION_STRING "scc_b200 0.1 (sm_100a)"

struct Params {
    Graph g;
    Work w;
    int t1, t2, lw;
    uint32_t tail_n;
    uint32_t *out;      // canonical labels (device, V entries) written at the end of the run, or nullptr
    uint32_t pass_cap;  // passes after which the run stops with SCC_ERR_NOT_CONVERGED (0: no cap)
    uint32_t hold;      // failure-detection test hook (GridExec::sync), 0: off
};

// Canonical labels of vertices tid+1, tid+1+n, ...: every vertex takes the
// smallest member id of its SCC, which the update passes fold into
// smin[representative] (or label[v] holds it itself, LBL_SELF).  Runs after the last pass barrier, so label and
// smin are final.  Four vertices per thread and round: their label loads,
// then their smin gathers, are issued back to back, so a thread waits on
// two memory latencies per four vertices instead of two per vertex.  The
// pointers carry no __restrict__: inside the SCC kernel label and smin were
// written by other CTAs of the same launch and must not be read through the
// non-coherent read-only path.
constexpr uint32_t LABEL_UNROLL = 4;

// A vertex whose state still carries both visited bits with range 0 is a
// member of the first pivot's SCC left marked by the lazy Slota update; its
// label is first_min.
// SKIP_RESIDUAL: vertices still carrying the residual solver's tag
// (FV|BV|(i+1)) are left out; the solver writes theirs.
template <bool SKIP_RESIDUAL = false>
__device__ __forceinline__ void canon_labels(const uint32_t *label, const uint32_t *smin, const uint32_t *st,
                                             uint32_t first_min, uint32_t *out, uint32_t V, uint32_t tid, uint32_t n)
{
    for (uint32_t v0 = tid + 1u; v0 <= V; v0 += LABEL_UNROLL * n) {
        uint32_t l[LABEL_UNROLL];
        bool skip[LABEL_UNROLL];
#pragma unroll
        for (uint32_t j = 0; j < LABEL_UNROLL; ++j) {
            const uint32_t v = v0 + j * n;
            l[j] = v <= V ? label[v] : 0xFFFFFFFFu;
            const uint32_t s = v <= V ? st[v] : DEAD;
            if (s == (FVB | BVB)) l[j] = LBL_SELF | first_min;
            skip[j] = SKIP_RESIDUAL && (s & (FVB | BVB)) == (FVB | BVB) && (s & RMASK) != 0u;
        }
#pragma unroll
        for (uint32_t j = 0; j < LABEL_UNROLL; ++j)
            l[j] = (l[j] & LBL_SELF) ? (l[j] & ~LBL_SELF) : (l[j] <= V ? smin[l[j]] : 0u);
#pragma unroll
        for (uint32_t j = 0; j < LABEL_UNROLL; ++j) {
            const uint32_t v = v0 + j * n;
            if (v <= V && !skip[j]) out[v - 1u] = l[j];
        }
    }
}

__device__ __forceinline__ void write_labels(const Work &w, uint32_t V, uint32_t *out, uint32_t tid, uint32_t n)
{
    canon_labels(w.label, w.smin, w.st, *(volatile const uint32_t *)&w.ctl->first_min, out, V, tid, n);
}

// ---------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------
constexpr int GRID_THREADS = 1024;
constexpr int BLOCK_THREADS = 1024;

// queues: staging queues of the launch (3 on the whole-GPU kernel, 2 on one CTA)
static size_t dyn_smem_bytes(uint32_t qcap, unsigned queues, int threads = 1024)
{
    return (BQ_HDR + queues * (size_t)(threads / 32) * qcap) * sizeof(uint32_t);
}

template <bool INSTR, bool HONG>
__global__ void __launch_bounds__(GRID_THREADS, 1) k_scc_grid(Params p)
{
    if (*(volatile int *)&p.w.ctl->error) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) p.w.ctl->t_start = gtimer();
    bq_init();
    GridExec<INSTR> ex{p.w.ctl, 0u, p.pass_cap, p.hold};
    Carry cy{0u, 0u, 0u};
    int rc = HONG ? hong_front(ex, p.g, p.w, p.t1, p.t2, p.lw, cy) : slota_front(ex, p.g, p.w, p.t1, p.lw, cy);
    if (rc == RUN_DONE) rc = HONG ? hong_loop(ex, p.g, p.w, cy, p.tail_n) : slota_peels(ex, p.g, p.w, cy, p.tail_n);
    if (rc == RUN_RESIDUAL) {
        // the live vertices fit one CTA's shared memory: CTA 0 solves them
        // while the other CTAs write every other vertex's label (every SCC
        // outside the residual is final here)
        if (blockIdx.x != 0) {
            if (p.out)
                canon_labels<true>(p.w.label, p.w.smin, p.w.st, *(volatile const uint32_t *)&p.w.ctl->first_min, p.out,
                                   p.g.V, (blockIdx.x - 1u) * blockDim.x + threadIdx.x, (gridDim.x - 1u) * blockDim.x);
            return;
        }
        res_solve(p.g, p.w, p.w.L[cy.lsel], cy.nL, p.w.Q[1][(cy.gl - 1u) & 1u], last_count(ex, C_BQ), p.w.ctl,
                  p.out);
        res_trace(p.w.ctl, cy.gl, cy.nL);
        if (threadIdx.x == 0) {
            p.w.ctl->tail_pass = cy.gl;
            p.w.ctl->nlive_tail = cy.nL;
            p.w.ctl->passes = cy.gl + 1u;
            // the labels are complete when the kernel ends (a failed solve leaves them to k_canon_write)
            if (p.out && !*(volatile int *)&p.w.ctl->error) p.w.ctl->labels_done = 1u;
        }
        return;
    }
    if (rc == RUN_SWITCH) {
        // the live set is small: CTA 0 finishes alone with block barriers
        if (blockIdx.x != 0) return;
        if (threadIdx.x == 0) { p.w.ctl->tail_pass = cy.gl; p.w.ctl->nlive_tail = cy.nL; }
        BlockExec<INSTR> bx{p.w.ctl, cy.gl, p.pass_cap};
        bx.reset_counters();
        if (HONG) hong_loop(bx, p.g, p.w, cy, 0u);
        else slota_peels(bx, p.g, p.w, cy, 0u);
        bx.gl = cy.gl;
        if (threadIdx.x == 0) p.w.ctl->passes = bx.gl;
        return;
    }
    if (ex.leader()) p.w.ctl->passes = ex.gl;
    if (rc == RUN_DONE && p.out) {
        // every CTA is still here: the grid writes the labels (after a switch
        // to CTA 0 alone, k_canon_write does)
        write_labels(p.w, p.g.V, p.out, ex.tid(), ex.nthr());
        if (ex.leader()) p.w.ctl->labels_done = 1u;
    }
}

template <bool INSTR, bool HONG>
__global__ void __launch_bounds__(BLOCK_THREADS, 1) k_scc_block(Params p)
{
    if (*(volatile int *)&p.w.ctl->error) return;
    if (threadIdx.x == 0) p.w.ctl->t_start = gtimer();
    bq_init();
    BlockExec<INSTR> ex{p.w.ctl, 0u, p.pass_cap};
    ex.reset_counters();
    Carry cy{0u, 0u, 0u};
    int rc = HONG ? hong_front(ex, p.g, p.w, p.t1, p.t2, p.lw, cy) : slota_front(ex, p.g, p.w, p.t1, p.lw, cy);
    if (rc == RUN_DONE) rc = HONG ? hong_loop(ex, p.g, p.w, cy, 0u) : slota_peels(ex, p.g, p.w, cy, 0u);
    if (threadIdx.x == 0) p.w.ctl->passes = ex.gl;
    if (rc == RUN_DONE && p.out) {
        write_labels(p.w, p.g.V, p.out, threadIdx.x, blockDim.x);
        if (threadIdx.x == 0) p.w.ctl->labels_done = 1u;
    }
}

// Canonical labels: every vertex takes the smallest member id of its SCC,
// which the update passes fold into smin[representative].
// Skipped when the SCC kernel already wrote them (ctl->labels_done).
__global__ void k_canon_write(const uint32_t *__restrict__ label, const uint32_t *__restrict__ smin,
                              const uint32_t *__restrict__ st, uint32_t *__restrict__ out, uint32_t V, const Ctl *ctl,
                              CtlReset r)
{
    if (blockIdx.x == 0 && r.next) {
        // the next run's control block, as the host would write it
        unsigned *wd = reinterpret_cast<unsigned *>(r.next);
        for (unsigned i = threadIdx.x; i < sizeof(Ctl) / 4u; i += blockDim.x) wd[i] = 0u;
        __syncthreads();
        if (threadIdx.x == 0) {
            r.next->first_min = 0xFFFFFFFFu;
            r.next->timeout_ns = r.timeout_ns;
            r.next->trace = r.trace;
            r.next->trace_cap = r.trace_cap;
            if (r.pivkey) *r.pivkey = 0ull;
        }
    }
    if (ctl && ctl->labels_done) return;
    canon_labels(label, smin, st, ctl ? ctl->first_min : 0xFFFFFFFFu, out, V, blockIdx.x * blockDim.x + threadIdx.x,
                 gridDim.x * blockDim.x);
}

// CTAs of 256 threads for k_canon_write: one round of LABEL_UNROLL vertices
// per thread covers V.
int canon_ctas(uint32_t V) { return (int)(((uint64_t)V + 256u * LABEL_UNROLL - 1u) / (256u * LABEL_UNROLL) + 1u); }

// ---------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------
namespace {

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return SCC_OK;
    if (e == cudaErrorMemoryAllocation) return SCC_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice ||
        e == cudaErrorInvalidDevice)
        return SCC_ERR_NO_DEVICE;
    return SCC_ERR_CUDA;
}

#define CK(call)                                  \
    do {                                          \
        cudaError_t _e = (call);                  \
        if (_e != cudaSuccess) {                  \
            ctx->last_cuda_error = (int)_e;       \
            return cuda_status(_e);               \
        }                                         \
    } while (0)

template <bool INSTR, bool HONG>
void *grid_kernel_ptr() { return (void *)k_scc_grid<INSTR, HONG>; }
template <bool INSTR, bool HONG>
void *block_kernel_ptr() { return (void *)k_scc_block<INSTR, HONG>; }

void *pick_grid(bool instr, bool hong)
{
    if (instr) return hong ? grid_kernel_ptr<true, true>() : grid_kernel_ptr<true, false>();
    return hong ? grid_kernel_ptr<false, true>() : grid_kernel_ptr<false, false>();
}
void *pick_block(bool instr, bool hong)
{
    if (instr) return hong ? block_kernel_ptr<true, true>() : block_kernel_ptr<true, false>();
    return hong ? block_kernel_ptr<false, true>() : block_kernel_ptr<false, false>();
}

}  // namespace

namespace {

// Offsets of the whole-graph workspace (all 256-byte aligned).
struct WsLayout {
    size_t st, label, stamp, smin, L0, L1, S0, S1, Q[4], H[4], piv, ctl, need, hcap;
};

WsLayout ws_layout(uint32_t V, uint32_t E)
{
    WsLayout o{};
    o.hcap = (size_t)E / CH + (size_t)E / HEAVY_T + 64;
    const size_t n1 = (size_t)V + 1;
    size_t need = 0;
    auto take = [&](size_t bytes) { size_t off = need; need = align_up(need + bytes, 256); return off; };
    o.st = take(n1 * 4); o.label = take(n1 * 4); o.stamp = take(n1 * 4); o.smin = take(n1 * 4);
    o.L0 = take(n1 * 4); o.L1 = take(n1 * 4);
    o.S0 = take(n1 * 4); o.S1 = take(n1 * 4);
    for (int i = 0; i < 4; i++) o.Q[i] = take(n1 * 4);
    for (int i = 0; i < 4; i++) o.H[i] = take(o.hcap * sizeof(uint2));
    o.piv = take((4 * n1 + 8) * 8);
    o.ctl = take(sizeof(Ctl));
    o.need = need;
    return o;
}

}  // namespace

size_t scc_ctx_ws_need(uint32_t V, uint32_t E) { return ws_layout(V, E).need; }

int scc_ctx_reserve(scc_context *ctx, uint32_t V, uint32_t E)
{
    const WsLayout o = ws_layout(V, E);
    const size_t need = o.need, hcap = o.hcap;
    const size_t o_st = o.st, o_label = o.label, o_stamp = o.stamp, o_smin = o.smin, o_L0 = o.L0, o_L1 = o.L1;
    const size_t *o_Q = o.Q, *o_H = o.H;
    const size_t o_piv = o.piv, o_ctl = o.ctl;
    if (need > ctx->ws_bytes) {
        if (ctx->ws) cudaFree(ctx->ws);
        ctx->ws = nullptr;
        ctx->ws_bytes = 0;
        cudaError_t e = cudaMalloc((void **)&ctx->ws, need);
        if (e != cudaSuccess) { ctx->last_cuda_error = (int)e; cudaGetLastError(); return SCC_ERR_OOM; }
        ctx->ws_bytes = need;
    }
    char *b = ctx->ws;
    Work &w = ctx->work;
    w.st = (uint32_t *)(b + o_st);
    w.label = (uint32_t *)(b + o_label);
    w.stamp = (uint32_t *)(b + o_stamp);
    w.smin = (uint32_t *)(b + o_smin);
    w.L[0] = (uint32_t *)(b + o_L0);
    w.L[1] = (uint32_t *)(b + o_L1);
    w.S[0] = (uint32_t *)(b + o.S0);
    w.S[1] = (uint32_t *)(b + o.S1);
    w.Q[0][0] = (uint32_t *)(b + o_Q[0]);
    w.Q[0][1] = (uint32_t *)(b + o_Q[1]);
    w.Q[1][0] = (uint32_t *)(b + o_Q[2]);
    w.Q[1][1] = (uint32_t *)(b + o_Q[3]);
    w.H[0][0] = (uint2 *)(b + o_H[0]);
    w.H[0][1] = (uint2 *)(b + o_H[1]);
    w.H[1][0] = (uint2 *)(b + o_H[2]);
    w.H[1][1] = (uint2 *)(b + o_H[3]);
    w.hcap = (uint32_t)std::min<size_t>(hcap, 0xFFFFFFFFu);
    w.pivkey = (unsigned long long *)(b + o_piv);
    w.ctl = (Ctl *)(b + o_ctl);
    return SCC_OK;
}

int sccb_csr_mirror(scc_context *ctx, uint32_t V, uint32_t E)
{
    size_t nv = (size_t)V + 2, ne = std::max<size_t>(E, 1);
    if (nv > ctx->capV) {
        cudaFree(ctx->dFr); cudaFree(ctx->dBr); cudaFree(ctx->dlab);
        ctx->dFr = ctx->dBr = ctx->dlab = nullptr; ctx->capV = 0;
        CK(cudaMalloc((void **)&ctx->dFr, nv * 4));
        CK(cudaMalloc((void **)&ctx->dBr, nv * 4));
        CK(cudaMalloc((void **)&ctx->dlab, nv * 4));
        ctx->capV = nv;
    }
    if (ne > ctx->capE) {
        cudaFree(ctx->dFc); cudaFree(ctx->dBc);
        ctx->dFc = ctx->dBc = nullptr; ctx->capE = 0;
        CK(cudaMalloc((void **)&ctx->dFc, ne * 4));
        CK(cudaMalloc((void **)&ctx->dBc, ne * 4));
        ctx->capE = ne;
    }
    return SCC_OK;
}

extern "C" const char *scc_version(void) { return SCC_VERSION_STRING; }

extern "C" const char *scc_status_string(int s)
{
    switch (s) {
    case SCC_OK: return "ok";
    case SCC_ERR_INVALID_ARG: return "invalid argument";
    case SCC_ERR_CUDA: return "CUDA runtime error";
    case SCC_ERR_OOM: return "Error: Not enough memory on GPU";
    case SCC_ERR_TOO_LARGE: return "graph too large (V above 2^28 - 2)";
    case SCC_ERR_NO_DEVICE: return "no usable CUDA device (sm_100a required)";
    case SCC_ERR_BUDGET: return "device memory budget exceeded";
    case SCC_ERR_IO: return "Error Reading graph file";
    case SCC_ERR_OVERFLOW: return "internal work list overflow";
    case SCC_ERR_NOT_CONVERGED: return "iteration cap reached before convergence";
    case SCC_ERR_TIMEOUT: return "grid barrier wait timed out";
    case SCC_ERR_BAD_GRAPH: return "malformed CSR (offsets or vertex ids)";
    default: return "unknown status";
    }
}

extern "C" int scc_create(int device, scc_context **out)
{
    if (!out) return SCC_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= 0) { cudaGetLastError(); return SCC_ERR_NO_DEVICE; }
    if (device < 0 || device >= n) return SCC_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return SCC_ERR_NO_DEVICE;
    if (prop.major != 10) return SCC_ERR_NO_DEVICE;
    scc_context *ctx = new (std::nothrow) scc_context();
    if (!ctx) return SCC_ERR_OOM;
    ctx->device = device;
    ctx->nsm = prop.multiProcessorCount;
    ctx->coop = prop.cooperativeLaunch;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost((void **)&ctx->hctl, sizeof(Ctl)) != cudaSuccess ||
        cudaEventCreate(&ctx->ev[0]) != cudaSuccess || cudaEventCreate(&ctx->ev[1]) != cudaSuccess ||
        cudaEventCreate(&ctx->ev[2]) != cudaSuccess || cudaEventCreate(&ctx->ev[3]) != cudaSuccess) {
        cudaGetLastError();
        scc_destroy(ctx);
        return SCC_ERR_CUDA;
    }
    *out = ctx;
    return SCC_OK;
}

extern "C" int scc_destroy(scc_context *ctx)
{
    if (!ctx) return SCC_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->up) cudaStreamSynchronize(ctx->up);
    cudaFree(ctx->ws);
    cudaFree(ctx->dFr); cudaFree(ctx->dFc); cudaFree(ctx->dBr); cudaFree(ctx->dBc); cudaFree(ctx->dlab);
    for (auto *p : ctx->tarc) cudaFree(p);
    cudaFree(ctx->ttmp); cudaFree(ctx->tctl); cudaFree(ctx->dtext); cudaFree(ctx->ctlb[0]);
    if (ctx->hctl) cudaFreeHost(ctx->hctl);
    cudaFree(ctx->dtrace);
    if (ctx->htrace) cudaFreeHost(ctx->htrace);
    for (int i = 0; i < 4; i++) if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
    for (auto e : ctx->upev) if (e) cudaEventDestroy(e);
    for (int i = 0; i < 2; i++) {
        if (ctx->stage_ev[i]) cudaEventDestroy(ctx->stage_ev[i]);
        if (ctx->hstage[i]) cudaFreeHost(ctx->hstage[i]);
    }
    if (ctx->up) cudaStreamDestroy(ctx->up);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SCC_OK;
}

// Raises the dynamic shared memory limit of kernel fn on the current device
// to max_bytes, once per (device, kernel), under one process-wide lock.  The
// limit only ever goes up and every caller passes the largest size any of
// its launches of fn can request, so a launch on one host thread can never
// find the limit lowered by another thread between its check and its launch.
int sccb_smem_limit(void *fn, size_t max_bytes)
{
    static std::mutex mu;
    struct Done { int dev; void *fn; };
    static Done done[256];
    static int ndone = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_CUDA; }
    std::lock_guard<std::mutex> lock(mu);
    for (int i = 0; i < ndone; i++)
        if (done[i].dev == dev && done[i].fn == fn) return SCC_OK;
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_bytes);
    if (e != cudaSuccess) { cudaGetLastError(); return cuda_status(e); }
    if (ndone < 256) done[ndone++] = Done{dev, fn};
    return SCC_OK;
}

// Largest dynamic shared memory of the plain-path kernels: the staging
// slice is at most 576 entries (scc_set_tuning "qcap") in three queues.
static size_t max_plain_smem() { return dyn_smem_bytes(576, 3); }

// Makes sure the kernel's dynamic shared memory limit covers every launch
// of it and returns the grid of its cooperative launch, computed once per
// (kernel, shared memory, CTA cap).  Returns 0 on failure.
static int prepare_kernel(scc_context *ctx, void *fn, size_t smem, int threads)
{
    if (smem > max_plain_smem() || sccb_smem_limit(fn, max_plain_smem()) != SCC_OK) return 0;
    for (int i = 0; i < ctx->n_prepared; i++) {
        const scc_context::Prepared &q = ctx->prepared[i];
        if (q.fn == fn && q.smem == smem && q.cap == ctx->max_blocks_per_sm) return q.nblocks;
    }
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (ctx->max_blocks_per_sm > 0) occ = std::min(occ, ctx->max_blocks_per_sm);
    const int nb = occ * ctx->nsm;
    if (nb > 0) {
        const int slot = ctx->n_prepared < 8 ? ctx->n_prepared++ : 7;
        ctx->prepared[slot] = scc_context::Prepared{fn, smem, ctx->max_blocks_per_sm, nb};
    }
    return nb;
}

// Counters and times of the run that ended with ctx->ev[3] (complete).
static int read_result(scc_context *ctx, scc_stats *stats)
{
    const Ctl &c = *ctx->hctl;
    if (stats) {
        stats->num_trim1 = c.n_trim1;
        stats->num_trim2 = c.n_trim2;
        stats->num_pivot = c.n_pivot;
        stats->num_sccs = c.n_trim1 + c.n_trim2 + c.n_pivot;
        stats->edges_scanned = c.t_edges;
        stats->vertex_visits = c.t_verts;
        stats->passes = c.passes;
        stats->outer_iters = c.outer;
        stats->tail_pass = c.tail_pass;
        stats->gpu_launches = ctx->pend_launches;
        stats->grid_blocks = ctx->pend_blocks;
        stats->used_block_path = ctx->pend_block_path;
        cudaEventElapsedTime(&stats->kernel_ms, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&stats->total_ms, ctx->ev[0], ctx->ev[3]);
        stats->error_where = c.where;
    }
    return c.error ? c.error : SCC_OK;
}

// scc_run and scc_run_async: everything up to the last copy of the run is
// enqueued on the stream; async returns there, scc_run waits and reads.
static int run_impl(scc_context *ctx, const scc_csr_view *gv, int algo, uint32_t flags, int warp_width,
                    uint32_t *labels_out, scc_stats *stats, void *stream_arg, bool async)
{
    if (!ctx || !gv) return SCC_ERR_INVALID_ARG;
    if (stats) memset(stats, 0, sizeof(*stats));
    if (async && !(flags & SCC_FLAG_DEVICE)) return SCC_ERR_INVALID_ARG;
    const bool hong = algo == SCC_ALGO_VHONG || algo == SCC_ALGO_WHONG;
    const bool warped = algo == SCC_ALGO_WHONG || algo == SCC_ALGO_WSLOTA;
    if (!hong && algo != SCC_ALGO_VSLOTA && algo != SCC_ALGO_WSLOTA) return SCC_ERR_INVALID_ARG;
    int lw = -1;
    if (warped) {
        switch (warp_width) {
        case 1: lw = 0; break;
        case 2: lw = 1; break;
        case 4: lw = 2; break;
        case 8: lw = 3; break;
        case 16: lw = 4; break;
        case 32: lw = 5; break;
        default: return SCC_ERR_INVALID_ARG;   // the reference silently skips the BFS (scc_WCC.cu:216-246)
        }
    }
    const uint32_t V = gv->num_vertices, E = gv->num_edges;
    if (V > SCC_MAX_VERTICES || E > SCC_MAX_EDGES) return SCC_ERR_TOO_LARGE;
    if (V == 0) return SCC_OK;
    // wHong / wSlota: the virtual-warp schedule (W lanes per frontier vertex,
    // the reference's fwd_warp<W>) pays when W > 1 and a vertex has W arcs
    // or more on average; otherwise most lanes idle (or one lane walks a
    // whole list) and the warp walk of the vertex drivers expands the same
    // frontiers faster (4096^2 grid: W = 8 4.92 -> 3.83 ms, W = 1 8.0 ->
    // 3.83 ms).  Results do not depend on the schedule.
    if (lw >= 0 && (ctx->warp_schedule == 2 ||
                    (ctx->warp_schedule == 0 && (lw == 0 || (uint64_t)E < ((uint64_t)V << lw)))))
        lw = -1;
    const bool derive = (flags & SCC_FLAG_DERIVE_REVERSE) != 0;
    if (!gv->Fr || (!derive && !gv->Br) || (E && (!gv->Fc || (!derive && !gv->Bc)))) return SCC_ERR_INVALID_ARG;
    const bool dev = (flags & SCC_FLAG_DEVICE) != 0;
    const bool instr = (flags & SCC_FLAG_INSTRUMENT) != 0;
    std::lock_guard<std::mutex> lock(ctx->mu);
    CK(cudaSetDevice(ctx->device));
    // NULL is the legacy default stream, as everywhere in CUDA (it is also
    // the handle a PyTorch "current stream" has unless the caller set one)
    cudaStream_t st = (cudaStream_t)stream_arg;
    int rc = scc_ctx_reserve(ctx, V, E);
    if (rc != SCC_OK) return rc;
    unsigned launches = 0;

    CK(cudaEventRecord(ctx->ev[0], st));
    Graph g{V, E, gv->Fr, gv->Fc, gv->Br, gv->Bc, 0u};
    uint32_t *dout = labels_out;
    if (!dev || derive) {
        rc = sccb_csr_mirror(ctx, V, E);
        if (rc != SCC_OK) return rc;
    }
    if (!dev) {
        CK(cudaMemcpyAsync(ctx->dFr, gv->Fr, ((size_t)V + 2) * 4, cudaMemcpyHostToDevice, st));
        if (!derive) CK(cudaMemcpyAsync(ctx->dBr, gv->Br, ((size_t)V + 2) * 4, cudaMemcpyHostToDevice, st));
        if (E && !derive) {   // with derive, Fc crosses inside sccb_derive_reverse, beside its first kernels
            CK(cudaMemcpyAsync(ctx->dFc, gv->Fc, (size_t)E * 4, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(ctx->dBc, gv->Bc, (size_t)E * 4, cudaMemcpyHostToDevice, st));
        }
        g.Fr = ctx->dFr; g.Fc = ctx->dFc; g.Br = ctx->dBr; g.Bc = ctx->dBc;
        dout = labels_out ? ctx->dlab : nullptr;
    } else if (derive) {
        g.Br = ctx->dBr; g.Bc = ctx->dBc;   // built below from the caller's forward CSR
    }
    if (!E) { g.Fc = g.Fc ? g.Fc : ctx->work.st; g.Bc = g.Bc ? g.Bc : ctx->work.st; }
    g.vec = ((((uintptr_t)g.Fr) | ((uintptr_t)g.Br)) & 15u) == 0u ? 1u : 0u;

    // control block: zeroed, then the timeout.  Two blocks alternate; the
    // label kernel of a run resets the other one for the next run, which
    // then needs no copy from the host (same timeout and trace settings).
    if (!ctx->ctlb[0]) {
        Ctl *b2 = nullptr;
        if (cudaMalloc((void **)&b2, 2 * sizeof(Ctl)) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_OOM; }
        ctx->ctlb[0] = b2;
        ctx->ctlb[1] = b2 + 1;
    }
    const int ci = ctx->ctl_next;
    ctx->ctl_next = ci ^ 1;
    const CtlReset init{ctx->ctlb[ci ^ 1], (unsigned long long)ctx->timeout_ms * 1000000ull, ctx->dtrace,
                        ctx->dtrace ? ctx->trace_cap : 0u, hong ? nullptr : ctx->work.pivkey};
    const bool ready = ctx->ctl_ready[ci] && ctx->ctl_made[ci].timeout_ns == init.timeout_ns &&
                       ctx->ctl_made[ci].trace == init.trace && ctx->ctl_made[ci].trace_cap == init.trace_cap;
    const bool piv_ready = ready && !hong && ctx->ctl_made[ci].pivkey == ctx->work.pivkey;
    ctx->ctl_ready[ci] = false;
    ctx->work.ctl = ctx->ctlb[ci];
    if (!ready) {
        memset(ctx->hctl, 0, sizeof(Ctl));
        ctx->hctl->first_min = 0xFFFFFFFFu;
        ctx->hctl->timeout_ns = init.timeout_ns;
        ctx->hctl->trace = init.trace;
        ctx->hctl->trace_cap = init.trace_cap;
        CK(cudaMemcpyAsync(ctx->work.ctl, ctx->hctl, sizeof(Ctl), cudaMemcpyHostToDevice, st));
    }
    if (derive) {
        // after the control block is zeroed: input errors found here stop the SCC kernel at its entry
        rc = sccb_derive_reverse(ctx, g.Fr, g.Fc, V, E, const_cast<uint32_t *>(g.Br), const_cast<uint32_t *>(g.Bc),
                                 ctx->work.ctl, st, dev ? nullptr : gv->Fc);
        if (rc != SCC_OK) return rc;
    }
    if (!piv_ready) CK(cudaMemsetAsync(ctx->work.pivkey, 0, hong ? (4 * ((size_t)V + 1) + 8) * 8 : 8, st));


    ctx->work.qcap = ctx->qcap;
    ctx->work.bu_k = ctx->bu_k;
    ctx->work.pull_lane = ctx->pull_lane;
    const size_t smem_block = dyn_smem_bytes(ctx->qcap, 2), smem_grid = dyn_smem_bytes(ctx->qcap, 3);
    Params p{g, ctx->work, (flags & SCC_FLAG_TRIM1) ? 1 : 0, (flags & SCC_FLAG_TRIM2) ? 1 : 0, lw, ctx->tail_vertices,
             dout, ctx->max_passes, ctx->hold_pass};
    bool use_block = (V <= ctx->block_max_vertices && E <= ctx->block_max_edges);
    if (flags & SCC_FLAG_FORCE_GRID) use_block = false;
    if (flags & SCC_FLAG_FORCE_BLOCK) use_block = true;
    if (!ctx->coop) use_block = true;
    int nblocks = 1;
    CK(cudaEventRecord(ctx->ev[1], st));
    if (use_block) {
        void *fn = pick_block(instr, hong);
        if (prepare_kernel(ctx, fn, smem_block, BLOCK_THREADS) <= 0) return SCC_ERR_CUDA;
        void *args[] = {&p};
        CK(cudaLaunchKernel(fn, dim3(1), dim3(BLOCK_THREADS), args, smem_block, st));
    } else {
        void *fn = pick_grid(instr, hong);
        nblocks = prepare_kernel(ctx, fn, smem_grid, GRID_THREADS);
        if (nblocks <= 0) return SCC_ERR_CUDA;
        void *args[] = {&p};
        CK(cudaLaunchCooperativeKernel(fn, dim3(nblocks), dim3(GRID_THREADS), args, smem_grid, st));
    }
    launches++;
    CK(cudaEventRecord(ctx->ev[2], st));
    if (dout) {
        k_canon_write<<<canon_ctas(V), 256, 0, st>>>(ctx->work.label, ctx->work.smin, ctx->work.st, dout, V,
                                                     ctx->work.ctl, init);
        launches += 1;
        CK(cudaGetLastError());
        ctx->ctl_made[ci ^ 1] = init;
        ctx->ctl_ready[ci ^ 1] = true;
        if (!dev) CK(cudaMemcpyAsync(labels_out, dout, (size_t)V * 4, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaMemcpyAsync(ctx->hctl, ctx->work.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    if (ctx->dtrace) CK(cudaMemcpyAsync(ctx->htrace, ctx->dtrace, (size_t)ctx->trace_cap * 16, cudaMemcpyDeviceToHost, st));
    CK(cudaEventRecord(ctx->ev[3], st));
    ctx->pend_launches = launches;
    ctx->pend_blocks = (uint32_t)nblocks;
    ctx->pend_block_path = use_block ? 1u : 0u;
    ctx->pending = true;
    if (async) return SCC_OK;
    CK(cudaStreamSynchronize(st));
    ctx->pending = false;
    return read_result(ctx, stats);
}

extern "C" int scc_run(scc_context *ctx, const scc_csr_view *gv, int algo, uint32_t flags, int warp_width,
                       uint32_t *labels_out, scc_stats *stats, void *stream_arg)
{
    return run_impl(ctx, gv, algo, flags, warp_width, labels_out, stats, stream_arg, false);
}

extern "C" int scc_run_async(scc_context *ctx, const scc_csr_view *gv, int algo, uint32_t flags, int warp_width,
                             uint32_t *labels_out, void *stream)
{
    return run_impl(ctx, gv, algo, flags, warp_width, labels_out, nullptr, stream, true);
}

extern "C" int scc_finish(scc_context *ctx, scc_stats *stats)
{
    if (!ctx) return SCC_ERR_INVALID_ARG;
    if (stats) memset(stats, 0, sizeof(*stats));
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!ctx->pending) return SCC_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess || cudaEventSynchronize(ctx->ev[3]) != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    ctx->pending = false;
    return read_result(ctx, stats);
}

extern "C" int scc_set_tuning(scc_context *ctx, const char *key, long long value)
{
    if (!ctx || !key) return SCC_ERR_INVALID_ARG;
    if (!strcmp(key, "tail_vertices")) ctx->tail_vertices = (uint32_t)value;
    else if (!strcmp(key, "block_max_vertices")) ctx->block_max_vertices = (uint32_t)value;
    else if (!strcmp(key, "block_max_edges")) ctx->block_max_edges = (uint32_t)value;
    else if (!strcmp(key, "timeout_ms")) ctx->timeout_ms = (uint32_t)value;
    else if (!strcmp(key, "max_blocks_per_sm")) ctx->max_blocks_per_sm = (int)value;
    else if (!strcmp(key, "bu_k")) ctx->bu_k = (uint32_t)value;
    else if (!strcmp(key, "warp_schedule")) {
        if (value < 0 || value > 2) return SCC_ERR_INVALID_ARG;
        ctx->warp_schedule = (int)value;
    }
    else if (!strcmp(key, "pull_lane")) {
        if (value < 1 || value > 1024) return SCC_ERR_INVALID_ARG;
        ctx->pull_lane = (uint32_t)value;
    }
    else if (!strcmp(key, "cluster_check")) ctx->cluster_check = value ? 1 : 0;
    else if (!strcmp(key, "max_passes")) ctx->max_passes = (uint32_t)value;
    else if (!strcmp(key, "test_withhold_arrival")) ctx->hold_pass = (uint32_t)value;
    else if (!strcmp(key, "qcap")) {
        if (value < 32 || value > 576) return SCC_ERR_INVALID_ARG;
        ctx->qcap = (uint32_t)value;
    } else if (!strcmp(key, "trace")) {
        // per-pass trace of the next runs: `value` passes (0 switches it off)
        std::lock_guard<std::mutex> lock(ctx->mu);
        cudaSetDevice(ctx->device);
        cudaFree(ctx->dtrace);
        cudaFreeHost(ctx->htrace);
        ctx->dtrace = nullptr;
        ctx->htrace = nullptr;
        ctx->trace_cap = 0;
        if (value > 0) {
            if (cudaMalloc((void **)&ctx->dtrace, (size_t)value * 16) != cudaSuccess ||
                cudaMallocHost((void **)&ctx->htrace, (size_t)value * 16) != cudaSuccess) {
                cudaGetLastError();
                return SCC_ERR_OOM;
            }
            ctx->trace_cap = (uint32_t)value;
        }
    } else return SCC_ERR_INVALID_ARG;
    return SCC_OK;
}

extern "C" int scc_get_trace(scc_context *ctx, uint64_t *out, uint32_t cap, uint32_t *n_out, uint64_t *t_start)
{
    if (!ctx || !n_out) return SCC_ERR_INVALID_ARG;
    uint32_t n = std::min<uint32_t>(ctx->hctl ? ctx->hctl->passes : 0u, ctx->trace_cap);
    if (out && ctx->htrace) memcpy(out, ctx->htrace, (size_t)std::min(n, cap) * 16);
    *n_out = n;
    if (t_start) *t_start = ctx->hctl ? ctx->hctl->t_start : 0;
    return SCC_OK;
}

// Launch sequence of the single-CTA path on caller-provided scratch (used by
// the no-allocation entry point in scc_noalloc.cu): the SCC kernel (which
// also validates the offsets) and the canonical-label kernel.  Allocates
// nothing.
int sccb_launch_block_path(const Graph &g, const Work &w, int t1, int t2, int lw, bool hong, uint32_t *dout,
                           cudaStream_t st, unsigned *launches)
{
    const size_t smem = dyn_smem_bytes(w.qcap, 2);
    void *fn = pick_block(false, hong);
    if (smem > max_plain_smem()) return SCC_ERR_INVALID_ARG;
    const int rc = sccb_smem_limit(fn, max_plain_smem());
    if (rc != SCC_OK) return rc;
    Params p{g, w, t1, t2, lw, 0u, nullptr, 0u, 0u};
    void *args[] = {&p};
    cudaError_t e = cudaLaunchKernel(fn, dim3(1), dim3(BLOCK_THREADS), args, smem, st);
    if (e != cudaSuccess) return cuda_status(e);
    k_canon_write<<<canon_ctas(g.V), 256, 0, st>>>(w.label, w.smin, w.st, dout, g.V, w.ctl, CtlReset{});
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
    *launches = 2;
    return SCC_OK;
}
