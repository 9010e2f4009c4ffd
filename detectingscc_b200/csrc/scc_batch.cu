// Batched form: thousands of independent graphs in one persistent launch.
//
// The graphs are uploaded once into one arena (packed CSR arrays).  One
// launch of k_scc_batch runs them all: every CTA takes the next graph from
// a work counter (graphs ordered largest first, so the long ones start
// early), re-carves its private scratch for that graph and runs the same
// driver code as the plain path with the single-CTA execution policy
// (BlockExec), then writes the graph's canonical labels and counters.  SCCs
// never cross graphs, so graphs need no coordination.  The launch (counter
// reset + kernel) is captured once into a CUDA graph and replayed.
//
// SCC_FLAG_BATCH_SEQUENTIAL runs the same graphs as per-graph plain calls
// (scc_run on device pointers into the arena, one after the other on one
// stream): the baseline the batched launch is measured against.
//
// Schedules (CTA size 128 / 256 / 512 / 1024 threads, staging slice size,
// cluster size and the vertex count from which a graph runs on a whole
// cluster) are picked by scc_batch_autotune, which times candidates on the
// batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "../../include/scc_b200.h"
#include "scc_internal.h"
#include "scc_phases.cuh"

#include <cooperative_groups.h>

using namespace sccb;

#include "scc_batch_internal.h"

namespace {

// Runs one graph with execution policy `ex` on the scratch slice `base`
// (every CTA of the policy calls it with the same arguments).
template <bool HONG, class Ex>
__device__ void batch_one(Ex &ex, const BatchParams &p, uint32_t gi, char *base, Work &s_w)
{
    const BatchGraph bg = p.graphs[gi];
    const unsigned long long t0 = gtimer();
    if (bg.V == 0u) {
        if (ex.leader()) {
            p.res[gi] = BatchRes{0ull, 0ull, 0ull, 0, 0, 0ull};
            if (p.done) {
                __threadfence_system();
                *(volatile unsigned *)&p.done[gi] = 1u;
            }
        }
        return;
    }
    Graph g{bg.V, bg.E, p.Fr + bg.off_r, p.Fc + bg.off_c, p.Br + bg.off_r, p.Bc + bg.off_c, p.vec};
    if (threadIdx.x == 0) {
        carve_work(base, bg.V, bg.E, HONG, &s_w);
        s_w.qcap = p.qcap;
        s_w.bu_k = p.bu_k;
        s_w.pull_lane = PULL_LANE;
    }
    __syncthreads();
    const Work &w = s_w;
    ex.ctl = w.ctl;
    // fresh control block and pivot table for this graph
    {
        uint32_t *c = reinterpret_cast<uint32_t *>(w.ctl);
        for (unsigned i = ex.tid(); i < sizeof(Ctl) / 4; i += ex.nthr()) c[i] = 0u;
        const uint32_t npk = HONG ? 4u * (bg.V + 1u) + 8u : 1u;
        for (uint32_t i = ex.tid(); i < npk; i += ex.nthr()) w.pivkey[i] = 0ull;
        ex.sync();
        if constexpr (!Ex::cluster) ex.reset_counters();   // this CTA's counter ring and error flag
        if (ex.leader()) {
            w.ctl->timeout_ns = p.timeout_ns;
            w.ctl->first_min = 0xFFFFFFFFu;
        }
        ex.sync();
    }
    ex.gl = 0u;
    Carry cy{0u, 0u, 0u};
    int rc = HONG ? hong_front(ex, g, w, p.t1, p.t2, p.lw, cy) : slota_front(ex, g, w, p.t1, p.lw, cy);
    if (rc == RUN_DONE) rc = HONG ? hong_loop(ex, g, w, cy, 0u) : slota_peels(ex, g, w, cy, 0u);
    ex.sync();   // the same error word in every CTA of the policy
    const int err = *(volatile int *)&w.ctl->error;
    if (!err) {
        uint32_t *o = p.out + bg.off_out;
        for (uint32_t v = ex.tid() + 1u; v <= bg.V; v += ex.nthr()) {
            const uint32_t l = w.label[v];
            o[v - 1u] = (l & LBL_SELF) ? (l & ~LBL_SELF) : (l <= bg.V ? w.smin[l] : 0u);
        }
    }
    if (ex.leader())
        p.res[gi] = BatchRes{w.ctl->n_trim1, w.ctl->n_trim2, w.ctl->n_pivot, err, w.ctl->where, gtimer() - t0};
    if (p.done) __threadfence_system();   // labels and result reach the host before the flag
    ex.sync();   // the slice is reused by the next graph
    if (p.done && ex.leader()) *(volatile unsigned *)&p.done[gi] = 1u;
}

// The first p.nbig graphs of p.order run one at a time on a whole cluster
// (when the launch has clusters), the rest one per CTA.  Counters:
// next[0] for cluster graphs, next[1] for CTA graphs.
// CL: the variant with the cluster loop, launched only when the batch has
// cluster graphs (kept apart so the common one-CTA-per-graph kernel does
// not carry the cluster path's registers).
template <int THREADS, bool HONG, bool CL>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_scc_batch(BatchParams p)
{
    __shared__ uint32_t s_k, s_kb;
    __shared__ Work s_w;   // per-graph carving, kept in shared memory rather than local memory
    bq_init();
    char *mine = p.scratch + (size_t)blockIdx.x * p.scratch_per_cta;
    if (CL && p.nbig) {
        const unsigned cr = cluster_rank(), cn = cluster_size();
        char *lead = p.scratch + (size_t)((blockIdx.x - cr) / p.lead_div) * p.scratch_per_cta;   // 1-D clusters
        for (;;) {
            if (cr == 0 && threadIdx.x == 0) s_kb = atomicAdd(&p.next[0], 1u);
            cluster_barrier();
            const uint32_t k = *cooperative_groups::this_cluster().map_shared_rank(&s_kb, 0);
            // check mode: every graph starts from a clean software barrier
            // word (all CTAs are past the previous graph here; a graph that
            // ended on a timed-out wait can leave the word mid-count)
            if (p.cbar && cr == 0 && threadIdx.x == 0) p.cbar[(blockIdx.x - cr) / cn] = 0u;
            cluster_barrier();   // rank 0 rewrites s_kb only after every CTA has read it
            if (k >= p.nbig) break;
            ClusterExec<false> ex{nullptr, 0u, cr, cn, p.cbar ? p.cbar + (blockIdx.x - cr) / cn : nullptr,
                                  p.timeout_ns, p.pass_cap, p.cbar ? p.hold : 0u};
            batch_one<HONG>(ex, p, p.order[k], lead, s_w);
        }
    }
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_k = p.nbig + atomicAdd(&p.next[1], 1u);
        __syncthreads();
        const uint32_t k = s_k;
        if (k >= p.n) return;
        BlockExec<false> ex{nullptr, 0u, p.pass_cap};
        batch_one<HONG>(ex, p, p.order[k], mine, s_w);
    }
}

template <int THREADS>
void *batch_kernel(bool hong, bool cl)
{
    if (cl) return hong ? (void *)k_scc_batch<THREADS, true, true> : (void *)k_scc_batch<THREADS, false, true>;
    return hong ? (void *)k_scc_batch<THREADS, true, false> : (void *)k_scc_batch<THREADS, false, false>;
}

void *pick_batch_kernel(int threads, bool hong, bool cl = false)
{
    switch (threads) {
    case 128: return batch_kernel<128>(hong, cl);
    case 256: return batch_kernel<256>(hong, cl);
    case 512: return batch_kernel<512>(hong, cl);
    default: return batch_kernel<1024>(hong, cl);
    }
}

// two staging queues per CTA (the batched graphs run on single CTAs and clusters)
size_t batch_smem(int threads, uint32_t qcap) { return (BQ_HDR + 2 * (size_t)(threads / 32) * qcap) * 4; }

}  // namespace

size_t sccb_batch_smem(int threads, uint32_t qcap) { return batch_smem(threads, qcap); }

int sccb_batch_ctas(int threads, uint32_t qcap, int nsm, uint32_t *out, int cluster)
{
    const size_t smem = batch_smem(threads, qcap);
    // the limit covers the largest staging slice a schedule may use (768
    // entries, capped at 200 KB), so batches, autotuning and server lanes on
    // other host threads never lower it under one another
    const size_t smem_max = std::min<size_t>(batch_smem(threads, 768), 200 * 1024);
    if (smem > smem_max) return SCC_ERR_INVALID_ARG;
    for (int h = 0; h < 4; h++) {
        void *fn = pick_batch_kernel(threads, (h & 1) != 0, h >= 2);
        if (sccb_smem_limit(fn, smem_max) != SCC_OK ||
            (cluster > 8 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
            cudaGetLastError();
            return SCC_ERR_CUDA;
        }
    }
    if (cluster <= 1) {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pick_batch_kernel(threads, true), threads, smem) !=
                cudaSuccess || occ <= 0) {
            cudaGetLastError();
            return SCC_ERR_CUDA;
        }
        *out = (uint32_t)(occ * nsm);
        return SCC_OK;
    }
    // clusters resident at once (a cluster sits inside one GPC)
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)cluster * (unsigned)nsm);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, pick_batch_kernel(threads, true, true), &cfg) != cudaSuccess || ncl <= 0) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    *out = (uint32_t)(ncl * cluster);
    return SCC_OK;
}

int sccb_batch_launch(const BatchParams &p, int threads, bool hong, uint32_t ncta, cudaStream_t st, int cluster)
{
    BatchParams q = p;
    void *args[] = {&q};
    cudaError_t e;
    if (cluster <= 1 || p.nbig == 0) {   // no cluster graphs: the one-CTA-per-graph kernel
        e = cudaLaunchKernel(pick_batch_kernel(threads, hong), dim3(ncta), dim3(threads), args,
                             batch_smem(threads, p.qcap), st);
    } else {
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)cluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(ncta);
        cfg.blockDim = dim3((unsigned)threads);
        cfg.dynamicSmemBytes = batch_smem(threads, p.qcap);
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelExC(&cfg, pick_batch_kernel(threads, hong, true), args);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    return SCC_OK;
}

// CTAs of a launch over n graphs: at most the resident CTAs, a whole number
// of clusters.
uint32_t sccb_launch_ctas(uint32_t resident, uint32_t n, uint32_t nbig, int cluster)
{
    const uint32_t cs = cluster > 1 ? (uint32_t)cluster : 1u;
    const unsigned long long want = (unsigned long long)nbig * cs + (n - nbig);
    unsigned long long c = std::min<unsigned long long>(resident, std::max<unsigned long long>(want, 1ull));
    c = (c + cs - 1) / cs * cs;
    if (c > resident) c = resident / cs * cs;
    return (uint32_t)std::max<unsigned long long>(c, cs);
}

// Processing order: graphs with at least big_vertices vertices first (they
// run on whole clusters), then the rest, each part largest first.
uint32_t sccb_order(const BatchGraph *g, uint32_t n, uint32_t big_vertices, int cluster, uint32_t *order,
                    const unsigned long long *cost)
{
    const bool use = cluster > 1;
    std::iota(order, order + n, 0u);
    auto big = [&](uint32_t i) { return use && g[i].V >= big_vertices; };
    auto w = [&](uint32_t i) { return cost ? cost[i] : (unsigned long long)g[i].E + g[i].V; };
    std::stable_sort(order, order + n, [&](uint32_t a, uint32_t c) {
        if (big(a) != big(c)) return big(a);
        return w(a) > w(c);
    });
    uint32_t nb = 0;
    while (nb < n && big(order[nb])) nb++;
    return nb;
}

struct scc_batch {
    scc_context *ctx = nullptr;
    uint32_t n = 0;
    unsigned long long sumV = 0, sumE = 0, sumR = 0;
    uint32_t maxV = 0, maxE = 0;
    uint32_t *dFr = nullptr, *dFc = nullptr, *dBr = nullptr, *dBc = nullptr, *dout = nullptr, *dorder = nullptr;
    BatchGraph *dgraphs = nullptr;
    std::vector<BatchGraph> hgraphs;
    BatchRes *dres = nullptr, *hres = nullptr;
    unsigned *dnext = nullptr;
    unsigned *dcbar = nullptr;       // per-cluster software barrier words (check mode)
    char *scratch = nullptr;
    size_t scratch_bytes = 0, scratch_per_cta = 0;
    uint32_t ncta = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int threads = 256;
    uint32_t qcap = 256;
    int cluster = 1;                 // CTAs per cluster (1: every graph on one CTA)
    uint32_t big_vertices = 16384;   // graphs with at least this many vertices run on a whole cluster
    uint32_t nbig = 0;
    // per-graph times of the last batched run, and whether the order follows them
    std::vector<unsigned long long> last_ns;
    bool by_cost = false;
    // captured launch
    cudaGraphExec_t gexec = nullptr;
    int g_algo = 0, g_w = 0, g_threads = 0, g_cluster = 0, g_check = 0;
    uint32_t g_flags = 0, g_qcap = 0, g_big = 0, g_cap = 0, g_hold = 0, g_timeout = 0;
};

static void batch_free(scc_batch *b)
{
    if (!b) return;
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    cudaFree(b->dFr); cudaFree(b->dFc); cudaFree(b->dBr); cudaFree(b->dBc); cudaFree(b->dout);
    cudaFree(b->dorder); cudaFree(b->dgraphs); cudaFree(b->dres); cudaFree(b->dnext); cudaFree(b->dcbar); cudaFree(b->scratch);
    if (b->hres) cudaFreeHost(b->hres);
    for (auto &e : b->ev) if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

// Processing order and cluster-graph count for the current cluster schedule.
static int batch_upload_order(scc_batch *b, int cluster, uint32_t big_vertices)
{
    std::vector<uint32_t> order(std::max<uint32_t>(b->n, 1u));
    const bool cost = b->by_cost && b->last_ns.size() == b->n;
    const uint32_t nb = sccb_order(b->hgraphs.data(), b->n, big_vertices, cluster, order.data(),
                                   cost ? b->last_ns.data() : nullptr);
    if (b->n && (cudaMemcpyAsync(b->dorder, order.data(), (size_t)b->n * 4, cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
                 cudaStreamSynchronize(b->stream) != cudaSuccess)) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    b->nbig = nb;
    return SCC_OK;
}

// Scratch for the CTAs of a schedule (grown on demand); sets b->ncta.
static int batch_reserve_scratch(scc_batch *b, int threads, uint32_t qcap, int cluster, uint32_t nbig)
{
    uint32_t resident = 0;
    int rc = sccb_batch_ctas(threads, qcap, b->ctx->nsm, &resident, cluster);
    if (rc != SCC_OK) return rc;
    const uint32_t ncta = sccb_launch_ctas(resident, b->n, nbig, cluster);
    const size_t need = (size_t)ncta * b->scratch_per_cta;
    if (need > b->scratch_bytes) {
        cudaFree(b->scratch);
        b->scratch = nullptr;
        b->scratch_bytes = 0;
        if (cudaMalloc((void **)&b->scratch, need) != cudaSuccess) {
            cudaGetLastError();
            return SCC_ERR_OOM;
        }
        b->scratch_bytes = need;
    }
    b->ncta = ncta;
    return SCC_OK;
}

extern "C" int scc_batch_create(scc_context *ctx, const scc_csr_view *graphs, uint32_t n, scc_batch **out)
{
    if (!ctx || !out || (n && !graphs)) return SCC_ERR_INVALID_ARG;
    *out = nullptr;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return SCC_ERR_NO_DEVICE;
    scc_batch *b = new (std::nothrow) scc_batch();
    if (!b) return SCC_ERR_OOM;
    b->ctx = ctx;
    b->n = n;
    b->hgraphs.resize(n);
    for (uint32_t i = 0; i < n; i++) {
        const scc_csr_view &g = graphs[i];
        if (g.num_vertices > SCC_MAX_VERTICES || g.num_edges > SCC_MAX_EDGES) { batch_free(b); return SCC_ERR_TOO_LARGE; }
        if (!g.Fr || !g.Br || (g.num_edges && (!g.Fc || !g.Bc))) { batch_free(b); return SCC_ERR_INVALID_ARG; }
        b->hgraphs[i] = BatchGraph{g.num_vertices, g.num_edges, b->sumR, b->sumE, b->sumV};
        b->sumR += (unsigned long long)g.num_vertices + 2;
        b->sumE += g.num_edges;
        b->sumV += g.num_vertices;
        b->maxV = std::max(b->maxV, g.num_vertices);
        b->maxE = std::max(b->maxE, g.num_edges);
    }
    // pad each packed array so every graph's offsets stay 16-byte aligned is not
    // required: 128-bit offset loads are only used when the batch is aligned
    int rc = SCC_OK;
    auto alloc = [&](void **p, size_t bytes) {
        if (rc != SCC_OK) return;
        if (cudaMalloc(p, std::max<size_t>(bytes, 16)) != cudaSuccess) { cudaGetLastError(); rc = SCC_ERR_OOM; }
    };
    alloc((void **)&b->dFr, b->sumR * 4);
    alloc((void **)&b->dBr, b->sumR * 4);
    alloc((void **)&b->dFc, b->sumE * 4);
    alloc((void **)&b->dBc, b->sumE * 4);
    alloc((void **)&b->dout, b->sumV * 4);
    alloc((void **)&b->dorder, (size_t)n * 4);
    alloc((void **)&b->dgraphs, (size_t)n * sizeof(BatchGraph));
    alloc((void **)&b->dres, (size_t)n * sizeof(BatchRes));
    alloc((void **)&b->dnext, 16);
    alloc((void **)&b->dcbar, 4096);
    if (rc == SCC_OK && cudaMemset(b->dcbar, 0, 4096) != cudaSuccess) rc = SCC_ERR_CUDA;
    if (rc == SCC_OK && cudaMallocHost((void **)&b->hres, std::max<size_t>((size_t)n * sizeof(BatchRes), 16)) != cudaSuccess)
        rc = SCC_ERR_OOM;
    if (rc == SCC_OK && (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
                         cudaEventCreate(&b->ev[0]) != cudaSuccess || cudaEventCreate(&b->ev[1]) != cudaSuccess))
        rc = SCC_ERR_CUDA;
    if (rc != SCC_OK) { cudaGetLastError(); batch_free(b); return rc; }
    for (uint32_t i = 0; i < n && rc == SCC_OK; i++) {
        const scc_csr_view &g = graphs[i];
        const BatchGraph &bg = b->hgraphs[i];
        if (cudaMemcpyAsync(b->dFr + bg.off_r, g.Fr, ((size_t)g.num_vertices + 2) * 4, cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
            cudaMemcpyAsync(b->dBr + bg.off_r, g.Br, ((size_t)g.num_vertices + 2) * 4, cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
            rc = SCC_ERR_CUDA;
        if (g.num_edges && rc == SCC_OK &&
            (cudaMemcpyAsync(b->dFc + bg.off_c, g.Fc, (size_t)g.num_edges * 4, cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
             cudaMemcpyAsync(b->dBc + bg.off_c, g.Bc, (size_t)g.num_edges * 4, cudaMemcpyHostToDevice, b->stream) != cudaSuccess))
            rc = SCC_ERR_CUDA;
    }
    if (rc == SCC_OK &&
        (cudaMemcpyAsync(b->dgraphs, b->hgraphs.data(), (size_t)n * sizeof(BatchGraph), cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
         cudaStreamSynchronize(b->stream) != cudaSuccess))
        rc = SCC_ERR_CUDA;
    if (rc != SCC_OK) { cudaGetLastError(); batch_free(b); return rc; }
    // largest graphs first (longest-processing-time order)
    rc = batch_upload_order(b, b->cluster, b->big_vertices);
    if (rc != SCC_OK) { batch_free(b); return rc; }
    b->scratch_per_cta = carve_work(nullptr, b->maxV, b->maxE, true, nullptr);
    rc = batch_reserve_scratch(b, b->threads, b->qcap, b->cluster, b->nbig);
    if (rc != SCC_OK) { batch_free(b); return rc; }
    *out = b;
    return SCC_OK;
}

extern "C" int scc_batch_destroy(scc_batch *b)
{
    if (!b) return SCC_ERR_INVALID_ARG;
    cudaSetDevice(b->ctx->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_free(b);
    return SCC_OK;
}

extern "C" int scc_batch_set_schedule(scc_batch *b, int threads, uint32_t qcap)
{
    if (!b || !(threads == 128 || threads == 256 || threads == 512 || threads == 1024) || qcap < 32 || qcap > 768)
        return SCC_ERR_INVALID_ARG;
    if (batch_smem(threads, qcap) > 200 * 1024) return SCC_ERR_INVALID_ARG;
    cudaSetDevice(b->ctx->device);
    int rc = batch_reserve_scratch(b, threads, qcap, b->cluster, b->nbig);
    if (rc != SCC_OK) return rc;
    b->threads = threads;
    b->qcap = qcap;
    return SCC_OK;
}

extern "C" int scc_batch_set_cluster(scc_batch *b, int cluster, uint32_t big_vertices)
{
    if (!b || !(cluster == 1 || cluster == 2 || cluster == 4 || cluster == 8 || cluster == 16)) return SCC_ERR_INVALID_ARG;
    cudaSetDevice(b->ctx->device);
    int rc = batch_upload_order(b, cluster, big_vertices);
    if (rc == SCC_OK) rc = batch_reserve_scratch(b, b->threads, b->qcap, cluster, b->nbig);
    if (rc != SCC_OK) {
        // back to the previous schedule
        batch_upload_order(b, b->cluster, b->big_vertices);
        batch_reserve_scratch(b, b->threads, b->qcap, b->cluster, b->nbig);
        return rc;
    }
    b->cluster = cluster;
    b->big_vertices = big_vertices;
    return SCC_OK;
}

extern "C" int scc_batch_get_cluster(scc_batch *b, int *cluster, uint32_t *big_vertices, uint32_t *num_cluster_graphs)
{
    if (!b) return SCC_ERR_INVALID_ARG;
    if (cluster) *cluster = b->cluster;
    if (big_vertices) *big_vertices = b->big_vertices;
    if (num_cluster_graphs) *num_cluster_graphs = b->nbig;
    return SCC_OK;
}

extern "C" int scc_batch_get_schedule(scc_batch *b, int *threads, uint32_t *qcap)
{
    if (!b) return SCC_ERR_INVALID_ARG;
    if (threads) *threads = b->threads;
    if (qcap) *qcap = b->qcap;
    return SCC_OK;
}

static int lw_of(int algo, int w)
{
    if (algo != SCC_ALGO_WHONG && algo != SCC_ALGO_WSLOTA) return -1;
    switch (w) {
    case 1: return 0;
    case 2: return 1;
    case 4: return 2;
    case 8: return 3;
    case 16: return 4;
    case 32: return 5;
    default: return -2;
    }
}

// Per-graph plain calls, one after the other: the baseline of the batched form.
static int batch_run_sequential(scc_batch *b, int algo, uint32_t flags, int w, scc_stats *stats)
{
    for (uint32_t i = 0; i < b->n; i++) {
        const BatchGraph &bg = b->hgraphs[i];
        scc_csr_view v{bg.V, bg.E, b->dFr + bg.off_r, b->dFc + bg.off_c, b->dBr + bg.off_r, b->dBc + bg.off_c};
        scc_stats st;
        int rc = scc_run(b->ctx, &v, algo, (flags & ~SCC_FLAG_BATCH_SEQUENTIAL) | SCC_FLAG_DEVICE, w,
                         b->dout + bg.off_out, &st, b->stream);
        b->hres[i] = BatchRes{st.num_trim1, st.num_trim2, st.num_pivot, rc, st.error_where,
                              (unsigned long long)(st.total_ms * 1e6)};
        if (stats) stats->gpu_launches += st.gpu_launches;
    }
    cudaEventRecord(b->ev[1], b->stream);
    cudaEventSynchronize(b->ev[1]);
    if (stats) cudaEventElapsedTime(&stats->kernel_ms, b->ev[0], b->ev[1]);
    return SCC_OK;
}

extern "C" int scc_batch_run(scc_batch *b, int algo, uint32_t flags, int warp_width, uint32_t *labels_out,
                             scc_batch_result *results, scc_stats *stats)
{
    if (!b) return SCC_ERR_INVALID_ARG;
    if (stats) memset(stats, 0, sizeof(*stats));
    const bool hong = algo == SCC_ALGO_VHONG || algo == SCC_ALGO_WHONG;
    if (!hong && algo != SCC_ALGO_VSLOTA && algo != SCC_ALGO_WSLOTA) return SCC_ERR_INVALID_ARG;
    const int lw = lw_of(algo, warp_width);
    if (lw == -2) return SCC_ERR_INVALID_ARG;
    if (cudaSetDevice(b->ctx->device) != cudaSuccess) return SCC_ERR_NO_DEVICE;
    cudaEventRecord(b->ev[0], b->stream);
    if (flags & SCC_FLAG_BATCH_SEQUENTIAL) {
        batch_run_sequential(b, algo, flags, warp_width, stats);
    } else {
        const uint32_t keyflags = flags & (SCC_FLAG_TRIM1 | SCC_FLAG_TRIM2);
        if (!b->gexec || b->g_algo != algo || b->g_flags != keyflags || b->g_w != warp_width ||
            b->g_threads != b->threads || b->g_qcap != b->qcap || b->g_cluster != b->cluster ||
            b->g_big != b->big_vertices || b->g_check != b->ctx->cluster_check || b->g_cap != b->ctx->max_passes ||
            b->g_hold != b->ctx->hold_pass || b->g_timeout != b->ctx->timeout_ms) {
            if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
            BatchParams p{b->dgraphs, b->dorder, b->n, b->dFr, b->dFc, b->dBr, b->dBc, 0u, b->dout, b->dres,
                          b->scratch, (unsigned long long)b->scratch_per_cta, b->dnext, b->nbig,
                          b->ctx->cluster_check && b->cluster > 1 ? b->dcbar : nullptr, 1u, nullptr, b->qcap, b->ctx->bu_k,
                          (flags & SCC_FLAG_TRIM1) ? 1 : 0, (flags & SCC_FLAG_TRIM2) ? 1 : 0, lw,
                          (unsigned long long)b->ctx->timeout_ms * 1000000ull, b->ctx->max_passes,
                          b->ctx->hold_pass};
            cudaGraph_t graph = nullptr;
            if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                cudaGetLastError();
                return SCC_ERR_CUDA;
            }
            cudaMemsetAsync(b->dnext, 0, 8, b->stream);
            sccb_batch_launch(p, b->threads, hong, b->ncta, b->stream, b->cluster);
            if (cudaStreamEndCapture(b->stream, &graph) != cudaSuccess ||
                cudaGraphInstantiate(&b->gexec, graph, 0) != cudaSuccess) {
                if (graph) cudaGraphDestroy(graph);
                cudaGetLastError();
                return SCC_ERR_CUDA;
            }
            cudaGraphDestroy(graph);
            b->g_algo = algo; b->g_flags = keyflags; b->g_w = warp_width;
            b->g_threads = b->threads; b->g_qcap = b->qcap; b->g_cluster = b->cluster; b->g_big = b->big_vertices;
            b->g_check = b->ctx->cluster_check;
            b->g_cap = b->ctx->max_passes;
            b->g_hold = b->ctx->hold_pass;
            b->g_timeout = b->ctx->timeout_ms;
        }
        if (cudaGraphLaunch(b->gexec, b->stream) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_CUDA; }
        cudaEventRecord(b->ev[1], b->stream);
        if (cudaMemcpyAsync(b->hres, b->dres, (size_t)b->n * sizeof(BatchRes), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess) {
            cudaGetLastError();
            return SCC_ERR_CUDA;
        }
        if (stats) stats->gpu_launches = 1;
    }
    if (labels_out && b->sumV &&
        cudaMemcpyAsync(labels_out, b->dout, b->sumV * 4, cudaMemcpyDeviceToHost, b->stream) != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_CUDA; }
    int first_err = SCC_OK;
    unsigned long long tot = 0;
    if (!(flags & SCC_FLAG_BATCH_SEQUENTIAL)) {
        b->last_ns.resize(b->n);
        for (uint32_t i = 0; i < b->n; i++) b->last_ns[i] = b->hres[i].ns;
    }
    for (uint32_t i = 0; i < b->n; i++) {
        const BatchRes &r = b->hres[i];
        if (results) results[i] = scc_batch_result{r.trim1 + r.trim2 + r.pivot, r.trim1, r.status, 0u};
        if (r.status && first_err == SCC_OK) first_err = r.status;
        tot += r.trim1 + r.trim2 + r.pivot;
    }
    if (stats) {
        stats->num_sccs = tot;
        stats->grid_blocks = (flags & SCC_FLAG_BATCH_SEQUENTIAL) ? 0u : b->ncta;
        if (!(flags & SCC_FLAG_BATCH_SEQUENTIAL)) cudaEventElapsedTime(&stats->kernel_ms, b->ev[0], b->ev[1]);
    }
    return first_err;
}

// Picks the CTA size and staging slice by timing every candidate on the
// batch itself (one untimed and two timed runs each), then, with that
// schedule, the cluster size and the vertex count from which graphs run on
// whole clusters.
extern "C" int scc_batch_autotune(scc_batch *b, int algo, uint32_t flags, int warp_width, int *best_threads,
                                  uint32_t *best_qcap, float *best_ms)
{
    if (!b) return SCC_ERR_INVALID_ARG;
    const uint32_t rflags = flags & ~SCC_FLAG_BATCH_SEQUENTIAL;
    auto time_it = [&](float *ms) -> int {
        scc_stats st;
        int rc = scc_batch_run(b, algo, rflags, warp_width, nullptr, nullptr, &st);
        if (rc != SCC_OK && rc < SCC_ERR_OVERFLOW) return rc;
        *ms = 0.f;
        for (int rep = 0; rep < 2; rep++) {
            scc_batch_run(b, algo, rflags, warp_width, nullptr, nullptr, &st);
            *ms += st.kernel_ms;
        }
        return SCC_OK;
    };
    const int cand_t[] = {128, 256, 512, 1024};
    const uint32_t cand_q[] = {64, 256};
    float best = 1e30f;
    int bt = b->threads;
    uint32_t bq = b->qcap;
    int rc = scc_batch_set_cluster(b, 1, b->big_vertices);
    if (rc != SCC_OK) return rc;
    for (int t : cand_t) {
        for (uint32_t q : cand_q) {
            if (scc_batch_set_schedule(b, t, q) != SCC_OK) continue;
            float ms = 0.f;
            rc = time_it(&ms);
            if (rc != SCC_OK) return rc;
            if (ms < best) { best = ms; bt = t; bq = q; }
        }
    }
    rc = scc_batch_set_schedule(b, bt, bq);
    if (rc != SCC_OK) return rc;
    int bc = 1;
    uint32_t bb = b->big_vertices;
    const int cand_c[] = {2, 4, 8};
    const uint32_t cand_b[] = {8192, 16384, 32768};
    for (int c : cand_c) {
        for (uint32_t v : cand_b) {
            if (scc_batch_set_cluster(b, c, v) != SCC_OK) continue;
            if (b->nbig == 0) continue;
            float ms = 0.f;
            rc = time_it(&ms);
            if (rc != SCC_OK) return rc;
            if (ms < best) { best = ms; bc = c; bb = v; }
        }
    }
    rc = scc_batch_set_cluster(b, bc, bb);
    if (rc != SCC_OK) return rc;
    // profile-guided order: longest-processing-time first by the graphs' own
    // times in a run with the chosen schedule (size is a poor proxy: a chain
    // of many small SCCs takes far longer than a random graph of its size)
    {
        float ms = 0.f;
        rc = time_it(&ms);   // leaves the per-graph times of its last run in last_ns
        if (rc != SCC_OK) return rc;
        b->by_cost = true;
        rc = batch_upload_order(b, b->cluster, b->big_vertices);
        if (rc != SCC_OK) return rc;
        float ms2 = 0.f;
        rc = time_it(&ms2);
        if (rc != SCC_OK) return rc;
        if (ms2 < best) {
            best = ms2;
        } else {
            b->by_cost = false;
            rc = batch_upload_order(b, b->cluster, b->big_vertices);
        }
    }
    if (best_threads) *best_threads = bt;
    if (best_qcap) *best_qcap = bq;
    if (best_ms) *best_ms = best / 2.f;
    return rc;
}

extern "C" int scc_batch_info(scc_batch *b, uint64_t *num_vertices, uint64_t *num_edges, uint32_t *num_graphs)
{
    if (!b) return SCC_ERR_INVALID_ARG;
    if (num_vertices) *num_vertices = b->sumV;
    if (num_edges) *num_edges = b->sumE;
    if (num_graphs) *num_graphs = b->n;
    return SCC_OK;
}
