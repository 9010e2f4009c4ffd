// scc_run_noalloc: the SCC decomposition without any device allocation.
//
// Some callers cannot call cudaMalloc at the time they need an SCC: a
// process whose device memory is entirely reserved up front by another
// allocator (a framework's caching pool, a serving process with a fixed
// memory budget), or a plugin whose host forbids allocating outside its own
// pool.  This entry point serves them: it runs the single-CTA SCC kernel
// (the same kernel scc_run uses for small graphs) on a fixed scratch area
// that lives in this file as a static __device__ array, so the caller only
// provides the device CSR and the device output buffer.
//
// Limits and behaviour:
//   * graphs up to NOALLOC_MAX_V vertices and NOALLOC_MAX_E edges; larger
//     graphs are rejected with SCC_ERR_TOO_LARGE before anything runs;
//   * the scratch array (NOALLOC_BYTES) is part of the module, so every GPU
//     that loads the library holds it until the process exits;
//   * on the first call on a device, with that device current, the call
//     looks up the device address of the array (cudaGetSymbolAddress) and
//     caches it per CUDA context (a context created later, e.g. after
//     cudaDeviceReset, gets its own lookup); make that first call before
//     any stream capture;
//   * flags other than SCC_FLAG_DEVICE (required), SCC_FLAG_TRIM1 and
//     SCC_FLAG_TRIM2 are rejected;
//   * every call shares the one array and overwrites it: calls whose work
//     overlaps on the GPU (different streams, threads) race and must be
//     serialised by the caller;
//   * the control block and pivot table are cleared on every call
//     (cudaMemsetAsync, which allocates nothing); no cudaMalloc, cudaFree,
//     events or library allocator is used.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/scc_b200.h"
#include "scc_device.cuh"

using namespace sccb;

int sccb_launch_block_path(const Graph &g, const Work &w, int t1, int t2, int lw, bool hong, uint32_t *dout,
                           cudaStream_t st, unsigned *launches);

namespace {

constexpr uint32_t NOALLOC_QCAP = 512;

constexpr size_t al256(size_t x) { return (x + 255) / 256 * 256; }

// Bytes the single-CTA kernel needs for a graph of V vertices and E edges
// (the same arrays scc_run sizes per graph: vertex state, labels, stamps,
// two live lists, four frontier queues, four heavy-chunk queues, the pivot
// table and the control block).
constexpr size_t scratch_bytes(size_t V, size_t E)
{
    return al256((V + 1) * 4) * 10 + al256((E / CH + E / HEAVY_T + 64) * 8) * 4 + al256((4 * (V + 1) + 8) * 8) +
           al256(sizeof(Ctl));
}

constexpr size_t NOALLOC_BYTES = scratch_bytes(SCC_NOALLOC_MAX_VERTICES, SCC_NOALLOC_MAX_EDGES);

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

std::mutex g_mu;

// Unique id of the calling thread's current CUDA context, 0 when there is
// none yet or the driver cannot tell.  The two driver entry points are
// fetched through the runtime, so the library needs no link-time libcuda.
unsigned long long current_ctx_id()
{
    using GetCurrent = int (*)(void **);
    using GetId = int (*)(void *, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool tried = false;
    if (!tried) {   // under g_mu
        tried = true;
        void *f = nullptr, *h = nullptr;
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &h, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess && f && h) {
            get_current = (GetCurrent)f;
            get_id = (GetId)h;
        }
        cudaGetLastError();
    }
    void *c = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&c) == 0 && c && get_id(c, &id) == 0) return id;
    return 0;
}

struct AddrEntry {
    unsigned long long ctx;
    void *addr;
};
constexpr int MAX_CTX = 64;
AddrEntry g_addr[MAX_CTX] = {};
int g_naddr = 0;

// Device address of the scratch array in the current context (looked up
// once per context: the first call on a device, with that device current).
// In host code the array's name is only a host-side stand-in; kernels must
// be given this address.
int scratch_address(char **out)
{
    std::lock_guard<std::mutex> lock(g_mu);
    unsigned long long id = current_ctx_id();
    if (id) {
        for (int i = 0; i < g_naddr; i++) {
            if (g_addr[i].ctx == id) {
                *out = (char *)g_addr[i].addr;
                return SCC_OK;
            }
        }
    }
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    if (!id) id = current_ctx_id();   // the lookup above made the primary context current
    if (id) g_addr[g_naddr < MAX_CTX ? g_naddr++ : (int)(id % MAX_CTX)] = AddrEntry{id, p};
    *out = (char *)p;
    return SCC_OK;
}

__global__ void k_noalloc_ctl_init(Ctl *c, unsigned long long timeout_ns)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        memset(c, 0, sizeof(Ctl));
        c->first_min = 0xFFFFFFFFu;
        c->timeout_ns = timeout_ns;
    }
}

}  // namespace

extern "C" int scc_run_noalloc(const scc_csr_view *gv, int algo, uint32_t flags, int warp_width,
                               uint32_t *labels_out, scc_stats *stats, void *stream)
{
    if (stats) memset(stats, 0, sizeof(*stats));
    if (!gv || !labels_out) return SCC_ERR_INVALID_ARG;
    if (!(flags & SCC_FLAG_DEVICE)) return SCC_ERR_INVALID_ARG;   // host inputs would need a device copy
    if (flags & ~(SCC_FLAG_DEVICE | SCC_FLAG_TRIM1 | SCC_FLAG_TRIM2)) return SCC_ERR_INVALID_ARG;
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
        default: return SCC_ERR_INVALID_ARG;
        }
    }
    const uint32_t V = gv->num_vertices, E = gv->num_edges;
    if (V > SCC_NOALLOC_MAX_VERTICES || E > SCC_NOALLOC_MAX_EDGES) return SCC_ERR_TOO_LARGE;
    if (V == 0) return SCC_OK;
    if (!gv->Fr || !gv->Br || (E && (!gv->Fc || !gv->Bc))) return SCC_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_NO_DEVICE;
    }
    char *base = nullptr;
    int rc = scratch_address(&base);
    if (rc != SCC_OK) return rc;

    // carve the scratch exactly as scratch_bytes() counts it
    const size_t n1 = (size_t)V + 1;
    const size_t hcap = (size_t)E / CH + (size_t)E / HEAVY_T + 64;
    size_t off = 0;
    auto take = [&](size_t bytes) { char *p = base + off; off += al256(bytes); return p; };
    Work w{};
    w.st = (uint32_t *)take(n1 * 4);
    w.label = (uint32_t *)take(n1 * 4);
    w.stamp = (uint32_t *)take(n1 * 4);
    w.smin = (uint32_t *)take(n1 * 4);
    w.L[0] = (uint32_t *)take(n1 * 4);
    w.L[1] = (uint32_t *)take(n1 * 4);
    w.S[0] = w.S[1] = nullptr;   // the single-CTA kernel keeps no shrinking scope
    w.Q[0][0] = (uint32_t *)take(n1 * 4);
    w.Q[0][1] = (uint32_t *)take(n1 * 4);
    w.Q[1][0] = (uint32_t *)take(n1 * 4);
    w.Q[1][1] = (uint32_t *)take(n1 * 4);
    w.H[0][0] = (uint2 *)take(hcap * 8);
    w.H[0][1] = (uint2 *)take(hcap * 8);
    w.H[1][0] = (uint2 *)take(hcap * 8);
    w.H[1][1] = (uint2 *)take(hcap * 8);
    w.hcap = (uint32_t)hcap;
    w.pivkey = (unsigned long long *)take((4 * n1 + 8) * 8);
    w.ctl = (Ctl *)take(sizeof(Ctl));
    w.qcap = NOALLOC_QCAP;
    w.bu_k = 2;
    w.pull_lane = PULL_LANE;
    if (off > NOALLOC_BYTES) return SCC_ERR_TOO_LARGE;

    cudaStream_t st = (cudaStream_t)stream;
    Graph g{V, E, gv->Fr, gv->Fc ? gv->Fc : w.st, gv->Br, gv->Bc ? gv->Bc : w.st,
            ((((uintptr_t)gv->Fr) | ((uintptr_t)gv->Br)) & 15u) == 0u ? 1u : 0u};
    k_noalloc_ctl_init<<<1, 32, 0, st>>>(w.ctl, 4000ull * 1000000ull);
    if (cudaMemsetAsync(w.pivkey, 0, hong ? (4 * n1 + 8) * 8 : 8, st) != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    unsigned launches = 0;
    rc = sccb_launch_block_path(g, w, (flags & SCC_FLAG_TRIM1) ? 1 : 0, (flags & SCC_FLAG_TRIM2) ? 1 : 0, lw, hong,
                                labels_out, st, &launches);
    if (rc != SCC_OK) return rc;
    Ctl c;
    if (cudaMemcpyAsync(&c, w.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    if (stats) {
        stats->num_trim1 = c.n_trim1;
        stats->num_trim2 = c.n_trim2;
        stats->num_pivot = c.n_pivot;
        stats->num_sccs = c.n_trim1 + c.n_trim2 + c.n_pivot;
        stats->passes = c.passes;
        stats->outer_iters = c.outer;
        stats->gpu_launches = launches + 1;
        stats->grid_blocks = 1;
        stats->used_block_path = 1;
        stats->error_where = c.where;
    }
    return c.error ? c.error : SCC_OK;
}
