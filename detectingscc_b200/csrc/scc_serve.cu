// Serving form: a request server with continuous batching under a
// device-memory budget.
//
// Requests (one host CSR each, plus a host buffer for its labels) are
// queued by scc_server_submit from any thread.  The server runs `lanes`
// worker threads, each with its own CUDA stream; a lane that is free takes
// whatever has arrived, in arrival order:
//   * a graph above `large_vertices` alone, run on the whole-GPU path
//     (scc_run with the lane's own context);
//   * otherwise every waiting small graph up to `max_graphs_per_batch`,
//     packed into the lane's arena and run by the batched kernel in one
//     launch.
// Lanes work concurrently, so requests that arrive while others are on the
// GPU are picked up by the next free lane and their work overlaps on the
// device.  Device memory held by all lanes (arenas, contexts) is kept under
// `budget_bytes`: a lane grows its arena only if the total stays within the
// budget, releasing idle lanes' memory first and otherwise waiting for a
// lane to finish; a request that cannot fit even alone is answered with
// SCC_ERR_BUDGET.  Each result carries its latency (submit to labels in host
// memory).  No counterpart in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
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
};

struct Lane {
    int id = 0;
    cudaStream_t stream = nullptr;
    scc_context *ctx = nullptr;        // whole-GPU path for large graphs
    size_t ctx_bytes = 0;
    // arena of the batched path
    uint32_t *dFr = nullptr, *dFc = nullptr, *dBr = nullptr, *dBc = nullptr, *dout = nullptr, *dorder = nullptr;
    BatchGraph *dgraphs = nullptr;
    BatchRes *dres = nullptr, *hres = nullptr;
    unsigned *dnext = nullptr;
    char *scratch = nullptr;
    size_t capR = 0, capE = 0, capV = 0, capN = 0, capScratch = 0;
    bool busy = false;
    std::thread th;
    size_t held() const
    {
        return ctx_bytes + (capR * 2 + capE * 2 + capV) * 4 + capN * (4 + sizeof(BatchGraph) + sizeof(BatchRes)) +
               capScratch + (dnext ? 256 : 0);
    }
};

}  // namespace

struct scc_server {
    int device = 0;
    int nsm = 0;
    scc_server_config cfg{};
    uint32_t ctas = 0;                   // resident CTAs of the batch kernel on the device
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req> pending;
    std::deque<scc_server_result> done;
    size_t held_total = 0;               // device bytes held by all lanes
    bool stop = false;
    uint64_t next_ticket = 1;
    std::vector<Lane *> lanes;
    uint64_t n_done = 0, n_rejected = 0;
};

namespace {

size_t csr_bytes(const scc_csr_view &g) { return 4 * (2 * ((size_t)g.num_vertices + 2) + 2 * (size_t)g.num_edges); }

void lane_free_arena(Lane *L)
{
    cudaFree(L->dFr); cudaFree(L->dFc); cudaFree(L->dBr); cudaFree(L->dBc); cudaFree(L->dout);
    cudaFree(L->dorder); cudaFree(L->dgraphs); cudaFree(L->dres); cudaFree(L->dnext); cudaFree(L->scratch);
    if (L->hres) cudaFreeHost(L->hres);
    L->dFr = L->dFc = L->dBr = L->dBc = L->dout = L->dorder = nullptr;
    L->dgraphs = nullptr; L->dres = L->hres = nullptr; L->dnext = nullptr; L->scratch = nullptr;
    L->capR = L->capE = L->capV = L->capN = L->capScratch = 0;
}

void lane_free_all(Lane *L)
{
    lane_free_arena(L);
    if (L->ctx) { scc_destroy(L->ctx); L->ctx = nullptr; }
    L->ctx_bytes = 0;
}

// Bytes the whole-GPU path holds for a graph (workspace + CSR mirror).
size_t large_bytes(const scc_csr_view &g)
{
    return carve_work(nullptr, g.num_vertices, g.num_edges, true, nullptr) + csr_bytes(g) +
           4 * ((size_t)g.num_vertices + 2);
}

struct Job {
    std::vector<Req> reqs;
    bool large = false;
    size_t sumR = 0, sumE = 0, sumV = 0;
    uint32_t maxV = 0, maxE = 0;
};

// Arena sizes a batch job needs (capacities only grow).
void job_arena_need(const scc_server *s, const Job &j, const Lane *L, size_t *R, size_t *E, size_t *V, size_t *N,
                    size_t *S)
{
    *R = std::max(L->capR, j.sumR);
    *E = std::max(L->capE, std::max<size_t>(j.sumE, 4));
    *V = std::max(L->capV, std::max<size_t>(j.sumV, 4));
    *N = std::max(L->capN, j.reqs.size());
    const size_t per = carve_work(nullptr, j.maxV, j.maxE, true, nullptr);
    const size_t ncta = std::min<size_t>(s->ctas, j.reqs.size());
    *S = std::max(L->capScratch, per * ncta);
}

size_t arena_bytes(size_t R, size_t E, size_t V, size_t N, size_t S)
{
    return (R * 2 + E * 2 + V) * 4 + N * (4 + sizeof(BatchGraph) + sizeof(BatchRes)) + S + 256;
}

int lane_grow_arena(Lane *L, size_t R, size_t E, size_t V, size_t N, size_t S)
{
    auto grow = [](void **p, size_t &cap, size_t need, size_t elem) -> bool {
        if (need <= cap && *p) return true;
        cudaFree(*p);
        *p = nullptr;
        if (cudaMalloc(p, need * elem) != cudaSuccess) { cudaGetLastError(); cap = 0; return false; }
        cap = need;
        return true;
    };
    size_t r1 = L->capR, r2 = L->capR, e1 = L->capE, e2 = L->capE, n1 = L->capN, n2 = L->capN, n3 = L->capN;
    bool ok = grow((void **)&L->dFr, r1, R, 4) && grow((void **)&L->dBr, r2, R, 4) &&
              grow((void **)&L->dFc, e1, E, 4) && grow((void **)&L->dBc, e2, E, 4) &&
              grow((void **)&L->dout, L->capV, V, 4) && grow((void **)&L->dorder, n1, N, 4) &&
              grow((void **)&L->dgraphs, n2, N, sizeof(BatchGraph)) && grow((void **)&L->dres, n3, N, sizeof(BatchRes)) &&
              grow((void **)&L->scratch, L->capScratch, S, 1);
    if (ok && !L->dnext) ok = cudaMalloc((void **)&L->dnext, 256) == cudaSuccess;
    if (ok && N > L->capN) {
        if (L->hres) cudaFreeHost(L->hres);
        L->hres = nullptr;
        ok = cudaMallocHost((void **)&L->hres, N * sizeof(BatchRes)) == cudaSuccess;
    }
    if (!ok) { cudaGetLastError(); lane_free_arena(L); return SCC_ERR_OOM; }
    L->capR = R; L->capE = E; L->capN = N;
    return SCC_OK;
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

// Runs one batch job on lane L (called without the lock).
int run_batch_job(scc_server *s, Lane *L, Job &j, std::vector<BatchRes> &out)
{
    const bool hong = s->cfg.algo == SCC_ALGO_VHONG || s->cfg.algo == SCC_ALGO_WHONG;
    const uint32_t n = (uint32_t)j.reqs.size();
    std::vector<BatchGraph> hg(n);
    unsigned long long r = 0, e = 0, v = 0;
    for (uint32_t i = 0; i < n; i++) {
        const scc_csr_view &g = j.reqs[i].g;
        hg[i] = BatchGraph{g.num_vertices, g.num_edges, r, e, v};
        r += (unsigned long long)g.num_vertices + 2;
        e += g.num_edges;
        v += g.num_vertices;
    }
    cudaStream_t st = L->stream;
    bool ok = true;
    for (uint32_t i = 0; i < n && ok; i++) {
        const scc_csr_view &g = j.reqs[i].g;
        ok = cudaMemcpyAsync(L->dFr + hg[i].off_r, g.Fr, ((size_t)g.num_vertices + 2) * 4, cudaMemcpyHostToDevice, st) == cudaSuccess &&
             cudaMemcpyAsync(L->dBr + hg[i].off_r, g.Br, ((size_t)g.num_vertices + 2) * 4, cudaMemcpyHostToDevice, st) == cudaSuccess &&
             (!g.num_edges ||
              (cudaMemcpyAsync(L->dFc + hg[i].off_c, g.Fc, (size_t)g.num_edges * 4, cudaMemcpyHostToDevice, st) == cudaSuccess &&
               cudaMemcpyAsync(L->dBc + hg[i].off_c, g.Bc, (size_t)g.num_edges * 4, cudaMemcpyHostToDevice, st) == cudaSuccess));
    }
    std::vector<uint32_t> order(n);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return (unsigned long long)hg[a].E + hg[a].V > (unsigned long long)hg[b].E + hg[b].V;
    });
    ok = ok && cudaMemcpyAsync(L->dgraphs, hg.data(), n * sizeof(BatchGraph), cudaMemcpyHostToDevice, st) == cudaSuccess &&
         cudaMemcpyAsync(L->dorder, order.data(), n * 4, cudaMemcpyHostToDevice, st) == cudaSuccess &&
         cudaMemsetAsync(L->dnext, 0, 4, st) == cudaSuccess;
    if (!ok) { cudaGetLastError(); return SCC_ERR_CUDA; }
    const uint32_t ncta = std::min<uint32_t>(s->ctas, n);
    BatchParams p{L->dgraphs, L->dorder, n, L->dFr, L->dFc, L->dBr, L->dBc, 0u, L->dout, L->dres, L->scratch,
                  (unsigned long long)carve_work(nullptr, j.maxV, j.maxE, true, nullptr), L->dnext,
                  s->cfg.qcap, 2u, (s->cfg.flags & SCC_FLAG_TRIM1) ? 1 : 0, (s->cfg.flags & SCC_FLAG_TRIM2) ? 1 : 0,
                  lw_of(s->cfg.algo, s->cfg.warp_width), 4000ull * 1000000ull};
    int rc = sccb_batch_launch(p, s->cfg.batch_threads, hong, ncta, st);
    if (rc != SCC_OK) return rc;
    ok = cudaMemcpyAsync(L->hres, L->dres, n * sizeof(BatchRes), cudaMemcpyDeviceToHost, st) == cudaSuccess;
    for (uint32_t i = 0; i < n && ok; i++)
        if (j.reqs[i].labels && hg[i].V)
            ok = cudaMemcpyAsync(j.reqs[i].labels, L->dout + hg[i].off_out, (size_t)hg[i].V * 4, cudaMemcpyDeviceToHost,
                                 st) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) { cudaGetLastError(); return SCC_ERR_CUDA; }
    out.assign(L->hres, L->hres + n);
    return SCC_OK;
}

// Takes the next job off the queue (lock held).
Job take_job(scc_server *s)
{
    Job j;
    const Req &f = s->pending.front();
    if (f.g.num_vertices > s->cfg.large_vertices) {
        j.large = true;
        j.reqs.push_back(f);
        s->pending.pop_front();
        return j;
    }
    while (!s->pending.empty() && j.reqs.size() < s->cfg.max_graphs_per_batch &&
           s->pending.front().g.num_vertices <= s->cfg.large_vertices) {
        const Req &q = s->pending.front();
        j.reqs.push_back(q);
        j.sumR += (size_t)q.g.num_vertices + 2;
        j.sumE += q.g.num_edges;
        j.sumV += q.g.num_vertices;
        j.maxV = std::max(j.maxV, q.g.num_vertices);
        j.maxE = std::max(j.maxE, q.g.num_edges);
        s->pending.pop_front();
    }
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
        size_t R = 0, E = 0, V = 0, N = 0, S = 0, cur = 0, grow = 0;
        bool rejected = false;
        for (;;) {
            // memory this job needs on this lane, and what the lane must grow by
            size_t target;
            if (j.large) {
                target = std::max(L->ctx_bytes, large_bytes(j.reqs[0].g)) +
                         arena_bytes(L->capR, L->capE, L->capV, L->capN, L->capScratch);
            } else {
                job_arena_need(s, j, L, &R, &E, &V, &N, &S);
                target = L->ctx_bytes + arena_bytes(R, E, V, N, S);
            }
            cur = L->held();
            grow = target > cur ? target - cur : 0;
            if (target > s->cfg.budget_bytes) {
                if (j.reqs.size() > 1) {
                    // run the first graph alone, give the others back in order
                    for (size_t i = j.reqs.size(); i-- > 1;) s->pending.push_front(j.reqs[i]);
                    const Req first = j.reqs[0];
                    j = Job{};
                    j.reqs.push_back(first);
                    j.sumR = (size_t)first.g.num_vertices + 2;
                    j.sumE = first.g.num_edges;
                    j.sumV = first.g.num_vertices;
                    j.maxV = first.g.num_vertices;
                    j.maxE = first.g.num_edges;
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
                    lane_free_all(o);
                    s->held_total -= h;
                    freed = true;
                    if (s->held_total + grow <= s->cfg.budget_bytes) break;
                }
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
        int rc = SCC_OK;
        std::vector<BatchRes> br;
        std::vector<scc_stats> ls;
        if (j.large) {
            if (!L->ctx) {
                rc = scc_create(s->device, &L->ctx);
                if (rc == SCC_OK) {
                    scc_set_tuning(L->ctx, "timeout_ms", 4000);
                }
            }
            scc_stats st{};
            if (rc == SCC_OK)
                rc = scc_run(L->ctx, &j.reqs[0].g, s->cfg.algo, s->cfg.flags & ~(SCC_FLAG_DEVICE | SCC_FLAG_BATCH_SEQUENTIAL),
                             s->cfg.warp_width, j.reqs[0].labels, &st, L->stream);
            ls.push_back(st);
            L->ctx_bytes = L->ctx ? L->ctx->ws_bytes + (L->ctx->capV * 3 + L->ctx->capE * 2) * 4 : 0;
        } else {
            rc = lane_grow_arena(L, R, E, V, N, S);
            if (rc == SCC_OK) rc = run_batch_job(s, L, j, br);
        }

        lk.lock();
        // settle the accounting to what the lane really holds now
        s->held_total = s->held_total - (cur + grow) + L->held();
        for (size_t i = 0; i < j.reqs.size(); i++) {
            if (rc != SCC_OK) {
                finish(s, j.reqs[i], rc, 0, 0, t_start, L->id);
            } else if (j.large) {
                finish(s, j.reqs[i], SCC_OK, ls[0].num_sccs, ls[0].num_trim1, t_start, L->id);
            } else {
                const BatchRes &b = br[i];
                finish(s, j.reqs[i], b.status, b.trim1 + b.trim2 + b.pivot, b.trim1, t_start, L->id);
            }
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
    if (!c.lanes) c.lanes = 4;
    if (!c.max_graphs_per_batch) c.max_graphs_per_batch = 512;
    if (!c.large_vertices) c.large_vertices = 65536;
    if (!c.batch_threads) c.batch_threads = 256;
    if (!c.qcap) c.qcap = 128;
    if (!c.algo) c.algo = SCC_ALGO_VSLOTA;
    if (!c.warp_width) c.warp_width = 1;
    if (c.lanes > 64 || lw_of(c.algo, c.warp_width) == -2 ||
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
    int rc = sccb_batch_ctas(c.batch_threads, c.qcap, s->nsm, &s->ctas);
    if (rc != SCC_OK) { delete s; return rc; }
    for (uint32_t i = 0; i < c.lanes; i++) {
        Lane *L = new Lane();
        L->id = (int)i;
        if (cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            delete L;
            rc = SCC_ERR_CUDA;
            break;
        }
        s->lanes.push_back(L);
    }
    if (rc != SCC_OK) {
        for (Lane *L : s->lanes) { cudaStreamDestroy(L->stream); delete L; }
        delete s;
        return rc;
    }
    for (Lane *L : s->lanes) L->th = std::thread(lane_main, s, L);
    *out = s;
    return SCC_OK;
}

extern "C" int scc_server_submit(scc_server *s, const scc_csr_view *g, uint32_t *labels_out, uint64_t *ticket)
{
    if (!s || !g || !ticket) return SCC_ERR_INVALID_ARG;
    if (g->num_vertices > SCC_MAX_VERTICES || g->num_edges > SCC_MAX_EDGES) return SCC_ERR_TOO_LARGE;
    if (!g->Fr || !g->Br || (g->num_edges && (!g->Fc || !g->Bc))) return SCC_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return SCC_ERR_INVALID_ARG;
    Req r{s->next_ticket++, *g, labels_out, now_ms()};
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
    for (Lane *L : s->lanes) {
        lane_free_all(L);
        cudaStreamDestroy(L->stream);
        delete L;
    }
    delete s;
    return SCC_OK;
}
