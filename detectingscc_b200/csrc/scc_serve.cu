// Serving form: a request server with continuous batching under a
// device-memory budget.
//
// Requests (one host CSR each, plus a host buffer for its labels) are
// queued by scc_server_submit from any thread.  The server runs `lanes`
// worker threads, each with its own CUDA stream; a lane that is free takes
// whatever has arrived, in arrival order:
//   * a graph above `large_vertices` alone, run by the batched kernel on one
//     thread-block cluster of `large_cluster` CTAs;
//   * otherwise every waiting small graph up to `max_graphs_per_batch`,
//     packed into the lane's arena and run by the batched kernel in one
//     launch (graphs of at least `big_vertices` vertices on clusters of
//     `cluster` CTAs, the rest one per CTA).
// Lanes work concurrently, so requests that arrive while others are on the
// GPU are picked up by the next free lane and their copies and kernels
// overlap on the device; no launch needs the whole GPU, so none waits for
// another lane's kernels to drain.  Device memory held by all lanes is kept
// under `budget_bytes`: a lane grows its arena only if the total stays
// within the budget, releasing idle lanes' memory first and otherwise
// waiting for a lane to finish; a request that cannot fit even alone is
// answered with SCC_ERR_BUDGET.  Each result carries its latency (submit to
// labels in host memory).  No counterpart in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <atomic>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <numeric>
#include <thread>
#include <vector>

#include "../../include/scc_b200.h"
#include "scc_batch_internal.h"
#include "scc_internal.h"

using namespace sccb;

namespace {

double now_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Req {
    uint64_t ticket;
    scc_csr_view g;
    uint32_t *labels;
    double t_submit;
    bool pinned;        // all four CSR arrays are page-locked (copied by DMA directly)
};

struct Lane {
    int id = 0;
    cudaStream_t stream = nullptr;
    // device arena (packed CSR, batch tables, per-CTA scratch), stream-ordered allocations
    uint32_t *dFr = nullptr, *dFc = nullptr, *dBr = nullptr, *dBc = nullptr, *dorder = nullptr;
    BatchGraph *dgraphs = nullptr;
    unsigned *dnext = nullptr;
    char *scratch = nullptr;
    size_t capR = 0, capE = 0, capN = 0, capScratch = 0;
    // page-locked host memory: pageable inputs, graph tables; labels, results
    // and completion flags, which the kernel writes directly
    char *hin = nullptr;
    uint32_t *hout = nullptr;
    BatchRes *hres = nullptr;
    unsigned *hdone = nullptr;
    char *htab = nullptr;              // graph table + processing order of a batch
    size_t capIn = 0, capOut = 0, capRes = 0, capDone = 0, capTab = 0;
    bool busy = false;
    std::thread th;
    // time spent per step (ms), printed at destroy when SCC_SERVE_PROFILE is set
    enum { P_GROW, P_UPLOAD, P_LAUNCH, P_WAIT, P_COPYOUT, P_KERNEL, P_N };
    double prof[P_N] = {};
    uint64_t njobs = 0, ngraphs = 0;
    cudaEvent_t k0 = nullptr, k1 = nullptr;
    size_t held() const
    {
        return (capR * 2 + capE * 2) * 4 + capN * (4 + sizeof(BatchGraph)) + capScratch + (dnext ? 256 : 0);
    }
};

}  // namespace

struct scc_server {
    int device = 0;
    int nsm = 0;
    scc_server_config cfg{};
    uint32_t ctas = 0;                   // resident CTAs of a small-graph launch (clusters of cfg.cluster)
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req> pending;
    std::deque<scc_server_result> done;
    size_t held_total = 0;               // device bytes held by all lanes
    bool stop = false;
    uint64_t next_ticket = 1;
    std::vector<Lane *> lanes;
    uint64_t n_done = 0, n_rejected = 0;
    uint64_t n_launches = 0;             // kernel launches made by the lanes (warm-up included)
    cudaMemPool_t pool = nullptr;        // the lanes' device arenas (keeps freed blocks for reuse)
};

namespace {

size_t grow_to(size_t cap, size_t need) { return need <= cap ? cap : std::max(need, cap + cap / 2); }

void lane_free_arena(Lane *L)
{
    cudaStream_t st = L->stream;
    void *ptrs[] = {L->dFr, L->dFc, L->dBr, L->dBc, L->dorder, L->dgraphs, L->dnext, L->scratch};
    for (void *q : ptrs)
        if (q) cudaFreeAsync(q, st);
    L->dFr = L->dFc = L->dBr = L->dBc = L->dorder = nullptr;
    L->dgraphs = nullptr; L->dnext = nullptr; L->scratch = nullptr;
    L->capR = L->capE = L->capN = L->capScratch = 0;
}

void lane_free_host(Lane *L)
{
    void *ptrs[] = {L->hin, L->hout, L->hres, L->hdone, L->htab};
    for (void *q : ptrs)
        if (q) cudaFreeHost(q);
    L->hin = nullptr; L->hout = nullptr; L->hres = nullptr; L->hdone = nullptr; L->htab = nullptr;
    L->capIn = L->capOut = L->capRes = L->capDone = L->capTab = 0;
}

struct Job {
    std::vector<Req> reqs;
    bool large = false;
    size_t sumR = 0, sumE = 0, sumV = 0, inBytes = 0;
    uint32_t maxV = 0, maxE = 0;
    uint32_t nbig = 0;      // graphs of a small job that run on whole clusters
};

// CTAs of the job's launch.
uint32_t job_ctas(const scc_server *s, const Job &j)
{
    if (j.large) return s->cfg.large_cluster;
    return sccb_launch_ctas(s->ctas, (uint32_t)j.reqs.size(), j.nbig, (int)s->cfg.cluster);
}

size_t csr_bytes(const scc_csr_view &g) { return 4 * (2 * ((size_t)g.num_vertices + 2) + 2 * (size_t)g.num_edges); }

// Arena capacities for a job (capacities only grow; growth is geometric).
struct Caps {
    size_t R, E, N, S;
};

Caps job_caps(const scc_server *s, const Job &j, const Lane *L, bool exact)
{
    auto g = [&](size_t cap, size_t need) { return exact ? std::max(cap, need) : grow_to(cap, need); };
    Caps c;
    c.R = g(L->capR, j.sumR);
    c.E = g(L->capE, std::max<size_t>(j.sumE, 4));
    c.N = g(L->capN, j.reqs.size());
    // one scratch slice per CTA, or per cluster for a large graph
    const size_t per = carve_work(nullptr, j.maxV, j.maxE, true, nullptr);
    const size_t slices = j.large ? 1 : job_ctas(s, j);
    c.S = g(L->capScratch, per * slices);
    return c;
}

size_t caps_bytes(const Caps &c)
{
    return (c.R * 2 + c.E * 2) * 4 + c.N * (4 + sizeof(BatchGraph)) + c.S + 256;
}

// Grows the arena to the capacities; stream-ordered frees and allocations on
// the lane's stream, so growing never waits for other lanes' kernels.
int lane_grow_arena(Lane *L, const Caps &c, cudaMemPool_t pool)
{
    cudaStream_t st = L->stream;
    auto grow = [&](void **p, size_t cap, size_t need, size_t elem) -> bool {
        if (need <= cap && *p) return true;
        if (*p) cudaFreeAsync(*p, st);
        *p = nullptr;
        if (cudaMallocFromPoolAsync(p, need * elem, pool, st) != cudaSuccess) { cudaGetLastError(); *p = nullptr; return false; }
        return true;
    };
    bool ok = grow((void **)&L->dFr, L->capR, c.R, 4) && grow((void **)&L->dBr, L->capR, c.R, 4) &&
              grow((void **)&L->dFc, L->capE, c.E, 4) && grow((void **)&L->dBc, L->capE, c.E, 4) &&
              grow((void **)&L->dorder, L->capN, c.N, 4) && grow((void **)&L->dgraphs, L->capN, c.N, sizeof(BatchGraph)) &&
              grow((void **)&L->scratch, L->capScratch, c.S, 1) && grow((void **)&L->dnext, 256, 256, 1);
    if (!ok) { lane_free_arena(L); return SCC_ERR_OOM; }
    L->capR = c.R; L->capE = c.E; L->capN = c.N; L->capScratch = c.S;
    return SCC_OK;
}

// Page-locked host memory large enough for the job (not budgeted: the
// budget is device memory).
int lane_grow_host(Lane *L, const Job &j)
{
    auto grow = [](void **p, size_t &cap, size_t need, size_t floor) -> bool {
        if (need <= cap && *p) return true;
        if (*p) cudaFreeHost(*p);
        *p = nullptr;
        need = std::max(grow_to(cap, need), floor);
        if (cudaMallocHost(p, need) != cudaSuccess) { cudaGetLastError(); cap = 0; return false; }
        cap = need;
        return true;
    };
    const size_t n = std::max<size_t>(j.reqs.size(), 1);
    bool ok = (j.inBytes == 0 || grow((void **)&L->hin, L->capIn, j.inBytes, 0)) &&
              grow((void **)&L->hout, L->capOut, std::max<size_t>(j.sumV, 1) * 4, 16u << 20) &&
              grow((void **)&L->hres, L->capRes, n * sizeof(BatchRes), 1024 * sizeof(BatchRes)) &&
              grow((void **)&L->hdone, L->capDone, n * 4, 4096) &&
              grow((void **)&L->htab, L->capTab, n * (sizeof(BatchGraph) + 4), 1024 * (sizeof(BatchGraph) + 4));
    return ok ? SCC_OK : SCC_ERR_OOM;
}

int lw_of(int algo, int w)
{
    if (algo != SCC_ALGO_WHONG && algo != SCC_ALGO_WSLOTA) return -1;
    switch (w) {
    case 1: return 0; case 2: return 1; case 4: return 2; case 8: return 3; case 16: return 4; case 32: return 5;
    default: return -2;
    }
}

void finish(scc_server *s, const Req &r, int status, uint64_t nscc, uint64_t ntrim1, double t_start, int lane)
{
    scc_server_result res{};
    res.ticket = r.ticket;
    res.status = status;
    res.num_vertices = r.g.num_vertices;
    res.num_sccs = nscc;
    res.num_trim1 = ntrim1;
    res.latency_ms = now_ms() - r.t_submit;
    res.queue_ms = t_start - r.t_submit;
    res.lane = lane;
    s->done.push_back(res);
}

// Enqueues the host->device copies of a job's CSR arrays into the lane's
// arena on the lane's stream: page-locked inputs straight from the caller's
// arrays, pageable ones through the lane's page-locked staging.
bool upload(Lane *L, const Job &j, std::vector<BatchGraph> &hg)
{
    const uint32_t n = (uint32_t)j.reqs.size();
    hg.resize(n);
    unsigned long long r = 0, e = 0, v = 0;
    size_t in_off = 0;
    cudaStream_t st = L->stream;
    bool ok = true;
    for (uint32_t i = 0; i < n && ok; i++) {
        const scc_csr_view &g = j.reqs[i].g;
        hg[i] = BatchGraph{g.num_vertices, g.num_edges, r, e, v};
        const size_t nr = ((size_t)g.num_vertices + 2) * 4, ne = (size_t)g.num_edges * 4;
        const uint32_t *src[4] = {g.Fr, g.Br, g.Fc, g.Bc};
        uint32_t *dst[4] = {L->dFr + r, L->dBr + r, L->dFc + e, L->dBc + e};
        const size_t len[4] = {nr, nr, ne, ne};
        for (int a = 0; a < 4 && ok; a++) {
            if (!len[a]) continue;
            const void *from = src[a];
            if (!j.reqs[i].pinned) {
                memcpy(L->hin + in_off, src[a], len[a]);
                from = L->hin + in_off;
                in_off += len[a];
            }
            ok = cudaMemcpyAsync(dst[a], from, len[a], cudaMemcpyHostToDevice, st) == cudaSuccess;
        }
        r += (unsigned long long)g.num_vertices + 2;
        e += g.num_edges;
        v += g.num_vertices;
    }
    return ok;
}

// Runs one job on lane L (called without s->mu): copies in, one launch of
// the batched kernel, which writes every graph's labels, result and
// completion flag into the lane's page-locked memory.  Each request is
// answered as soon as its own graph is done, while the launch goes on with
// the others.  Returns SCC_OK, or an error for the requests not answered.
int run_job(scc_server *s, Lane *L, Job &j, double t_start, std::vector<char> &answered)
{
    const bool hong = s->cfg.algo == SCC_ALGO_VHONG || s->cfg.algo == SCC_ALGO_WHONG;
    const uint32_t n = (uint32_t)j.reqs.size();
    std::vector<BatchGraph> hg;
    cudaStream_t st = L->stream;
    double t0 = now_ms();
    bool ok = upload(L, j, hg);
    // graph table and processing order through page-locked staging
    BatchGraph *tg = (BatchGraph *)L->htab;
    uint32_t *order = (uint32_t *)(L->htab + (size_t)n * sizeof(BatchGraph));
    std::copy(hg.begin(), hg.end(), tg);
    const int cluster = j.large ? (int)s->cfg.large_cluster : (int)s->cfg.cluster;
    const uint32_t nbig = sccb_order(tg, n, j.large ? 0u : s->cfg.big_vertices, cluster, order);
    memset(L->hdone, 0, (size_t)n * 4);
    ok = ok && cudaMemcpyAsync(L->dgraphs, tg, n * sizeof(BatchGraph), cudaMemcpyHostToDevice, st) == cudaSuccess &&
         cudaMemcpyAsync(L->dorder, order, n * 4, cudaMemcpyHostToDevice, st) == cudaSuccess &&
         cudaMemsetAsync(L->dnext, 0, 8, st) == cudaSuccess;
    if (!ok) { cudaGetLastError(); return SCC_ERR_CUDA; }
    j.nbig = nbig;
    const uint32_t ncta = job_ctas(s, j);
    BatchParams p{L->dgraphs, L->dorder, n, L->dFr, L->dFc, L->dBr, L->dBc, 0u, L->hout, L->hres, L->scratch,
                  (unsigned long long)carve_work(nullptr, j.maxV, j.maxE, true, nullptr), L->dnext, nbig, nullptr,
                  j.large ? (uint32_t)cluster : 1u, L->hdone, s->cfg.qcap, 2u, (s->cfg.flags & SCC_FLAG_TRIM1) ? 1 : 0,
                  (s->cfg.flags & SCC_FLAG_TRIM2) ? 1 : 0, lw_of(s->cfg.algo, s->cfg.warp_width),
                  4000ull * 1000000ull, 0u, 0u};
    double t1 = now_ms();
    L->prof[Lane::P_UPLOAD] += t1 - t0;
    cudaEventRecord(L->k0, st);
    int rc = sccb_batch_launch(p, s->cfg.batch_threads, hong, ncta, st, cluster);
    cudaEventRecord(L->k1, st);
    if (rc == SCC_OK) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->n_launches++;
    }
    L->prof[Lane::P_LAUNCH] += now_ms() - t1;
    if (rc != SCC_OK) return rc;
    // answer requests as their flags come up
    std::vector<uint32_t> left(n), ready;
    std::iota(left.begin(), left.end(), 0u);
    volatile unsigned *flag = L->hdone;
    for (;;) {
        const cudaError_t q = cudaEventQuery(L->k1);   // sampled before the flags
        if (q != cudaSuccess && q != cudaErrorNotReady) { cudaGetLastError(); return SCC_ERR_CUDA; }
        ready.clear();
        size_t keep = 0;
        for (uint32_t i : left) {
            if (flag[i]) ready.push_back(i);
            else left[keep++] = i;
        }
        left.resize(keep);
        if (!ready.empty()) {
            std::atomic_thread_fence(std::memory_order_acquire);
            const double tc = now_ms();
            for (uint32_t i : ready)
                if (j.reqs[i].labels && hg[i].V)
                    memcpy(j.reqs[i].labels, L->hout + hg[i].off_out, (size_t)hg[i].V * 4);
            L->prof[Lane::P_COPYOUT] += now_ms() - tc;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                for (uint32_t i : ready) {
                    const BatchRes &b = L->hres[i];
                    finish(s, j.reqs[i], b.status, b.trim1 + b.trim2 + b.pivot, b.trim1, t_start, L->id);
                    answered[i] = 1;
                    s->n_done++;
                }
            }
            s->cv_done.notify_all();
        }
        if (left.empty()) break;
        if (q == cudaSuccess) return SCC_ERR_CUDA;      // launch ended without these graphs' flags
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_CUDA; }
    L->prof[Lane::P_WAIT] += now_ms() - t1;
    float kms = 0.f;
    if (cudaEventElapsedTime(&kms, L->k0, L->k1) == cudaSuccess) L->prof[Lane::P_KERNEL] += kms;
    cudaGetLastError();
    return SCC_OK;
}

// Takes the next job off the queue (lock held).
Job take_job(scc_server *s)
{
    Job j;
    auto add = [&](const Req &q) {
        j.reqs.push_back(q);
        j.sumR += (size_t)q.g.num_vertices + 2;
        j.sumE += q.g.num_edges;
        j.sumV += q.g.num_vertices;
        j.maxV = std::max(j.maxV, q.g.num_vertices);
        j.maxE = std::max(j.maxE, q.g.num_edges);
        if (!q.pinned) j.inBytes += csr_bytes(q.g);
        if (s->cfg.cluster > 1 && q.g.num_vertices >= s->cfg.big_vertices) j.nbig++;
    };
    const Req &f = s->pending.front();
    if (f.g.num_vertices > s->cfg.large_vertices) {
        j.large = true;
        add(f);
        s->pending.pop_front();
        return j;
    }
    while (!s->pending.empty() && j.reqs.size() < s->cfg.max_graphs_per_batch &&
           s->pending.front().g.num_vertices <= s->cfg.large_vertices) {
        add(s->pending.front());
        s->pending.pop_front();
    }
    return j;
}

Job single(const scc_server *s, const Req &q)
{
    Job j;
    j.reqs.push_back(q);
    j.large = q.g.num_vertices > s->cfg.large_vertices;
    j.sumR = (size_t)q.g.num_vertices + 2;
    j.sumE = q.g.num_edges;
    j.sumV = q.g.num_vertices;
    j.maxV = q.g.num_vertices;
    j.maxE = q.g.num_edges;
    j.inBytes = q.pinned ? 0 : csr_bytes(q.g);
    j.nbig = (s->cfg.cluster > 1 && q.g.num_vertices >= s->cfg.big_vertices) ? 1u : 0u;
    return j;
}

void lane_main(scc_server *s, Lane *L)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty(); });
        if (s->pending.empty()) {
            if (s->stop) break;
            continue;
        }
        Job j = take_job(s);
        L->busy = true;   // nobody frees this lane's memory while it plans and runs
        Caps caps{};
        size_t cur = 0, grow = 0;
        bool rejected = false;
        for (;;) {
            // device memory this job needs on this lane
            cur = L->held();
            caps = job_caps(s, j, L, false);
            size_t target = caps_bytes(caps);
            if (s->held_total + (target > cur ? target - cur : 0) > s->cfg.budget_bytes) {
                caps = job_caps(s, j, L, true);      // no headroom for geometric growth
                target = caps_bytes(caps);
            }
            grow = target > cur ? target - cur : 0;
            // what the job needs on an empty lane
            Lane empty;
            const size_t alone = caps_bytes(job_caps(s, j, &empty, true));
            if (alone > s->cfg.budget_bytes) {
                if (j.reqs.size() > 1) {
                    // run the first graph alone, give the others back in order
                    for (size_t i = j.reqs.size(); i-- > 1;) s->pending.push_front(j.reqs[i]);
                    j = single(s, j.reqs[0]);
                    continue;
                }
                finish(s, j.reqs[0], SCC_ERR_BUDGET, 0, 0, now_ms(), L->id);
                s->n_rejected++;
                s->n_done++;
                rejected = true;
                break;
            }
            if (s->held_total + grow <= s->cfg.budget_bytes) break;
            // release idle lanes' memory first, otherwise wait for a lane to finish
            bool freed = false;
            for (Lane *o : s->lanes) {
                if (o != L && !o->busy && o->held() > 0) {
                    size_t h = o->held();
                    lane_free_arena(o);
                    cudaStreamSynchronize(o->stream);
                    s->held_total -= h;
                    freed = true;
                    if (s->held_total + grow <= s->cfg.budget_bytes) break;
                }
            }
            if (freed) cudaMemPoolTrimTo(s->pool, 0);   // give the freed blocks back to the device
            if (!freed && cur > 0 && s->held_total + caps_bytes(job_caps(s, j, &empty, true)) - cur <= s->cfg.budget_bytes) {
                // this lane's own arena is in the way of an exact-size one
                lane_free_arena(L);
                cudaStreamSynchronize(L->stream);
                cudaMemPoolTrimTo(s->pool, 0);
                s->held_total -= cur;
                freed = true;
            }
            if (!freed) s->cv_done.wait(lk);
        }
        if (rejected) {
            L->busy = false;
            s->cv_done.notify_all();
            continue;
        }
        s->held_total += grow;
        lk.unlock();

        const double t_start = now_ms();
        std::vector<char> answered(j.reqs.size(), 0);
        int rc = lane_grow_arena(L, caps, s->pool);
        if (rc == SCC_OK) rc = lane_grow_host(L, j);
        L->prof[Lane::P_GROW] += now_ms() - t_start;
        L->njobs++;
        L->ngraphs += j.reqs.size();
        if (rc == SCC_OK) rc = run_job(s, L, j, t_start, answered);

        lk.lock();
        // settle the accounting to what the lane really holds now
        s->held_total = s->held_total - (cur + grow) + L->held();
        for (size_t i = 0; i < j.reqs.size(); i++) {
            if (answered[i]) continue;
            finish(s, j.reqs[i], rc != SCC_OK ? rc : SCC_ERR_CUDA, 0, 0, t_start, L->id);
            s->n_done++;
        }
        L->busy = false;
        s->cv_done.notify_all();
    }
}

}  // namespace

extern "C" int scc_server_create(int device, const scc_server_config *cfg, scc_server **out)
{
    if (!out) return SCC_ERR_INVALID_ARG;
    *out = nullptr;
    scc_server_config c{};
    if (cfg) c = *cfg;
    if (!c.budget_bytes) c.budget_bytes = 120ull * 1000 * 1000 * 1000;
    if (!c.lanes) c.lanes = 8;
    if (!c.max_graphs_per_batch) c.max_graphs_per_batch = 512;
    if (!c.large_vertices) c.large_vertices = 65536;
    if (!c.batch_threads) c.batch_threads = 1024;
    if (!c.qcap) c.qcap = 256;
    if (!c.algo) c.algo = SCC_ALGO_VSLOTA;
    if (!c.warp_width) c.warp_width = 1;
    if (!c.cluster) c.cluster = 4;
    if (!c.big_vertices) c.big_vertices = 16384;
    if (!c.large_cluster) c.large_cluster = 16;
    auto cl_ok = [](uint32_t x) { return x == 1 || x == 2 || x == 4 || x == 8 || x == 16; };
    if (!cl_ok(c.cluster) || !cl_ok(c.large_cluster)) return SCC_ERR_INVALID_ARG;
    if (c.lanes > 64 || lw_of(c.algo, c.warp_width) == -2 || c.qcap < 32 || c.qcap > 768 ||
        !(c.batch_threads == 128 || c.batch_threads == 256 || c.batch_threads == 512 || c.batch_threads == 1024) ||
        (c.algo != SCC_ALGO_VHONG && c.algo != SCC_ALGO_VSLOTA && c.algo != SCC_ALGO_WHONG && c.algo != SCC_ALGO_WSLOTA))
        return SCC_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) { cudaGetLastError(); return SCC_ERR_NO_DEVICE; }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return SCC_ERR_NO_DEVICE;
    cudaSetDevice(device);
    scc_server *s = new (std::nothrow) scc_server();
    if (!s) return SCC_ERR_OOM;
    s->device = device;
    s->nsm = prop.multiProcessorCount;
    s->cfg = c;
    int rc = sccb_batch_ctas(c.batch_threads, c.qcap, s->nsm, &s->ctas, (int)c.cluster);
    // the largest cluster the device can hold for large graphs (at most the one asked for)
    uint32_t big_res = 0;
    while (rc == SCC_OK && (sccb_batch_ctas(c.batch_threads, c.qcap, s->nsm, &big_res, (int)s->cfg.large_cluster) != SCC_OK ||
                            big_res < s->cfg.large_cluster)) {
        cudaGetLastError();
        if (s->cfg.large_cluster == 1) { rc = SCC_ERR_CUDA; break; }
        s->cfg.large_cluster /= 2;
    }
    if (rc != SCC_OK) { delete s; return rc; }
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = device;
    if (cudaMemPoolCreate(&s->pool, &pp) != cudaSuccess) { cudaGetLastError(); delete s; return SCC_ERR_CUDA; }
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    // A lane's allocation never waits on another lane's stream to reuse
    // memory that lane freed (such a wait would tie the lanes together).
    int no = 0;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolReuseAllowInternalDependencies, &no);
    // Reserve memory in the pool up front (1 GiB per lane, at most half the
    // budget): growing an arena then takes cached memory instead of new
    // device allocations, which took up to a second under load and stalled
    // every lane behind them.
    {
        const size_t warm = std::min<size_t>((size_t)c.lanes << 30, c.budget_bytes / 2);
        void *w = nullptr;
        if (warm && cudaMallocFromPoolAsync(&w, warm, s->pool, 0) == cudaSuccess) {
            cudaFreeAsync(w, 0);
            cudaStreamSynchronize(0);
        }
        cudaGetLastError();
    }
    for (uint32_t i = 0; i < c.lanes && rc == SCC_OK; i++) {
        Lane *L = new Lane();
        L->id = (int)i;
        s->lanes.push_back(L);
        if (cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&L->k0) != cudaSuccess || cudaEventCreate(&L->k1) != cudaSuccess) {
            cudaGetLastError();
            rc = SCC_ERR_CUDA;
        }
        // page-locked memory for a full batch of typical graphs up front
        Job typical;
        typical.reqs.resize(c.max_graphs_per_batch);
        typical.sumV = 16u << 20;
        if (rc == SCC_OK) rc = lane_grow_host(L, typical);
    }
    if (rc != SCC_OK) {
        for (Lane *L : s->lanes) {
            lane_free_host(L);
            if (L->stream) cudaStreamDestroy(L->stream);
            if (L->k0) cudaEventDestroy(L->k0);
            if (L->k1) cudaEventDestroy(L->k1);
            delete L;
        }
        cudaMemPoolDestroy(s->pool);
        delete s;
        return rc;
    }
    for (Lane *L : s->lanes) L->th = std::thread(lane_main, s, L);
    *out = s;
    return SCC_OK;
}

// A host range is page-locked (registered or cudaMallocHost'd) if CUDA
// reports it as host memory.
static bool is_pinned(const void *p)
{
    if (!p) return true;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return a.type == cudaMemoryTypeHost;
}

extern "C" int scc_server_submit(scc_server *s, const scc_csr_view *g, uint32_t *labels_out, uint64_t *ticket)
{
    if (!s || !g || !ticket) return SCC_ERR_INVALID_ARG;
    if (g->num_vertices > SCC_MAX_VERTICES || g->num_edges > SCC_MAX_EDGES) return SCC_ERR_TOO_LARGE;
    if (!g->Fr || !g->Br || (g->num_edges && (!g->Fc || !g->Bc))) return SCC_ERR_INVALID_ARG;
    const bool pinned = is_pinned(g->Fr) && is_pinned(g->Br) && is_pinned(g->Fc) && is_pinned(g->Bc);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return SCC_ERR_INVALID_ARG;
    Req r{s->next_ticket++, *g, labels_out, now_ms(), pinned};
    *ticket = r.ticket;
    s->pending.push_back(r);
    s->cv_work.notify_one();
    return SCC_OK;
}

extern "C" int scc_server_poll(scc_server *s, scc_server_result *out, uint32_t cap, uint32_t *n_out, int wait_ms)
{
    if (!s || !n_out || (cap && !out)) return SCC_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
    uint32_t n = 0;
    while (n < cap && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    *n_out = n;
    return SCC_OK;
}

extern "C" int scc_server_info(scc_server *s, uint64_t *pending, uint64_t *completed, uint64_t *held_bytes,
                               uint64_t *rejected)
{
    if (!s) return SCC_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (pending) *pending = s->pending.size();
    if (completed) *completed = s->n_done;
    if (held_bytes) *held_bytes = s->held_total;
    if (rejected) *rejected = s->n_rejected;
    return SCC_OK;
}

extern "C" int scc_server_launches(scc_server *s, uint64_t *launches)
{
    if (!s || !launches) return SCC_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *launches = s->n_launches;
    return SCC_OK;
}

extern "C" int scc_server_destroy(scc_server *s)
{
    if (!s) return SCC_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (Lane *L : s->lanes)
        if (L->th.joinable()) L->th.join();
    cudaSetDevice(s->device);
    if (getenv("SCC_SERVE_PROFILE")) {
        for (Lane *L : s->lanes)
            fprintf(stderr,
                    "lane %d: jobs %llu graphs %llu | ms grow %.1f upload %.1f launch %.1f wait %.1f "
                    "copyout %.1f | gpu kernel %.1f\n",
                    L->id, (unsigned long long)L->njobs, (unsigned long long)L->ngraphs, L->prof[Lane::P_GROW],
                    L->prof[Lane::P_UPLOAD], L->prof[Lane::P_LAUNCH], L->prof[Lane::P_WAIT],
                    L->prof[Lane::P_COPYOUT], L->prof[Lane::P_KERNEL]);
    }
    for (Lane *L : s->lanes) {
        cudaStreamSynchronize(L->stream);
        lane_free_arena(L);
        cudaStreamSynchronize(L->stream);   // the stream-ordered frees
        lane_free_host(L);
        cudaStreamDestroy(L->stream);
        cudaEventDestroy(L->k0);
        cudaEventDestroy(L->k1);
        delete L;
    }
    cudaMemPoolDestroy(s->pool);
    delete s;
    return SCC_OK;
}
