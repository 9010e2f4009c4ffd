// Host-side context of the engine (CUDA translation units only).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "scc_device.cuh"

constexpr unsigned UPLOAD_CHUNKS = 8;   // pieces of a host-to-device upload beside the reverse build

struct scc_context {
    int device = 0;
    int nsm = 0;
    int coop = 0;
    int last_cuda_error = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // upload of the forward targets beside the reverse-CSR build
    cudaStream_t up = nullptr;
    cudaEvent_t upev[UPLOAD_CHUNKS + 1] = {};
    sccb::Ctl *hctl = nullptr;   // pinned copy of the control block

    // device workspace (grows to the largest graph run so far)
    char *ws = nullptr;
    size_t ws_bytes = 0;
    sccb::Work work{};

    // device mirror of host CSR inputs
    uint32_t *dFr = nullptr, *dFc = nullptr, *dBr = nullptr, *dBc = nullptr, *dlab = nullptr;
    size_t capV = 0, capE = 0;

    // reverse CSR built on the device (SCC_FLAG_DERIVE_REVERSE) and GTgraph
    // text parsed on the device: the radix sorts' storage
    uint32_t *tarc[3] = {nullptr, nullptr, nullptr};   // arc-sized sort buffers
    void *ttmp = nullptr;               // digit histograms and scan sums
    sccb::Ctl *tctl = nullptr;          // error word of scc_derive_reverse / scc_load_graph_device
    size_t tcapE = 0, ttmp_bytes = 0;
    // two control blocks used in turn; made[i] records how block i was last
    // reset by a label kernel (ready[i]: not used since)
    sccb::Ctl *ctlb[2] = {nullptr, nullptr};
    int ctl_next = 0;
    bool ctl_ready[2] = {false, false};
    sccb::CtlReset ctl_made[2] = {};
    // the last run's launch facts, read back by scc_finish after scc_run_async
    bool pending = false;
    unsigned pend_launches = 0, pend_blocks = 0, pend_block_path = 0;
    char *dtext = nullptr;              // GTgraph text parsed on the device
    size_t text_cap = 0;
    char *hstage[2] = {nullptr, nullptr};            // page-locked file staging (scc_load_graph_device)
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};

    // tuning
    uint32_t tail_vertices = 1024;       // CTA 0 finishes alone at or below this live count
    uint32_t block_max_vertices = 16384; // graphs up to this size run on one CTA
    uint32_t block_max_edges = 262144;
    uint32_t timeout_ms = 4000;          // bound on any single grid-barrier wait
    int max_blocks_per_sm = 0;           // 0 = occupancy limit
    uint32_t qcap = 320;                 // per-warp staging slice entries (up to 3 queues x 32 warps in shared memory;
                                         // larger slices shrink the L1 data cache and slow the gathers)
    uint32_t bu_k = 2;                   // bottom-up BFS step when frontier edges > bu_k * scope (0 = off)
    int warp_schedule = 0;               // wHong/wSlota first search: 0 auto, 1 virtual warps, 2 warp walk
    uint32_t pull_lane = 4;              // bottom-up step: list length a lane tests alone (4: 2 % faster
                                         // than 32 on R-MAT scale 22, plain and permuted ids)
    int cluster_check = 0;               // batched launches: bounded software cluster barriers (check mode)
    uint32_t max_passes = 0;             // a run stops with SCC_ERR_NOT_CONVERGED after this many passes (0: no cap)
    uint32_t hold_pass = 0;              // failure-detection test hook: k + 1 = one CTA withholds its barrier
                                         // arrival at pass k (grid launches; batched launches in check mode)

    // grid size of the cooperative launch (occupancy x SMs) per kernel and
    // shared memory size, computed once
    struct Prepared { void *fn; size_t smem; int cap; int nblocks; };
    Prepared prepared[8] = {};
    int n_prepared = 0;

    // optional per-pass trace
    unsigned long long *dtrace = nullptr, *htrace = nullptr;
    uint32_t trace_cap = 0;

    std::mutex mu;
};

int scc_ctx_reserve(scc_context *ctx, uint32_t V, uint32_t E);
// Builds Br and Bc (device) from Fr (device) and Fc on stream st; errors in
// the input are raised in ctl.  Allocates its temporaries in ctx.  With hFc
// set, Fc is still in host memory and is copied to dFc here, in pieces that
// overlap the first kernels of the build.
int sccb_derive_reverse(scc_context *ctx, const uint32_t *dFr, const uint32_t *dFc, uint32_t V, uint32_t E,
                        uint32_t *dBr, uint32_t *dBc, sccb::Ctl *ctl, cudaStream_t st, const uint32_t *hFc);
// Device CSR arrays of the context (grown on demand): host inputs are copied
// there, scc_load_graph_device builds graphs there.
int sccb_csr_mirror(scc_context *ctx, uint32_t V, uint32_t E);
// Bytes of the workspace scc_ctx_reserve allocates for a graph.
size_t scc_ctx_ws_need(uint32_t V, uint32_t E);
// Raises kernel fn's dynamic shared memory limit on the current device to
// max_bytes once (process-wide lock); returns an scc_status.
int sccb_smem_limit(void *fn, size_t max_bytes);
