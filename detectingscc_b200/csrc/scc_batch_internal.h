// Device-side description of a packed set of graphs, shared by the batched
// form (scc_batch.cu) and the request server (scc_serve.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

struct BatchGraph {
    uint32_t V, E;
    unsigned long long off_r;   // into the packed Fr / Br arrays (V+2 entries per graph)
    unsigned long long off_c;   // into the packed Fc / Bc arrays
    unsigned long long off_out; // into the packed label output (V entries per graph)
};

struct BatchRes {
    unsigned long long trim1, trim2, pivot;
    int status, where;
    unsigned long long ns;      // time the graph took on its CTA or cluster (%globaltimer)
};

struct BatchParams {
    const BatchGraph *graphs;
    const uint32_t *order;      // processing order (largest first)
    uint32_t n;
    const uint32_t *Fr, *Fc, *Br, *Bc;
    uint32_t vec;
    uint32_t *out;
    BatchRes *res;
    char *scratch;              // ncta slices of scratch_per_cta bytes
    unsigned long long scratch_per_cta;
    unsigned *next;             // work counters next[0] (cluster graphs), next[1] (CTA graphs), zero before the launch
    uint32_t nbig;              // the first nbig graphs of order run on whole clusters
    unsigned *cbar;             // per-cluster software barrier counters (check mode), or nullptr
    uint32_t lead_div;          // a cluster graph uses slice (rank-0 CTA index) / lead_div: 1, or the
                                // cluster size when every graph of the launch is a cluster graph
    unsigned *done;             // optional per-graph completion flags (page-locked host memory): set to 1
                                // after the graph's labels and result are visible to the host
    uint32_t qcap, bu_k;
    int t1, t2, lw;
    unsigned long long timeout_ns;
    uint32_t pass_cap;          // per graph: passes after which the graph fails with SCC_ERR_NOT_CONVERGED (0: none)
    uint32_t hold;              // check mode: failure-detection test hook (ClusterExec::barrier), 0: off
};

// Shared memory of the batch kernel for a CTA size and staging slice.
size_t sccb_batch_smem(int threads, uint32_t qcap);
// Resident CTAs of the batch kernel on a device with nsm SMs, launched in
// clusters of `cluster` CTAs (1: no clusters; above 8 needs the non-portable
// cluster size, which this sets).
int sccb_batch_ctas(int threads, uint32_t qcap, int nsm, uint32_t *out, int cluster = 1);
// Launch of the batch kernel (the caller zeroes p.next[0..1] first).
int sccb_batch_launch(const BatchParams &p, int threads, bool hong, uint32_t ncta, cudaStream_t st, int cluster = 1);
// CTAs of a launch: at most `resident`, a whole number of clusters.
uint32_t sccb_launch_ctas(uint32_t resident, uint32_t n, uint32_t nbig, int cluster);
// Processing order (cluster graphs first, each part longest first: by cost[i]
// when given, measured times of an earlier run, else by V + E); returns nbig.
uint32_t sccb_order(const BatchGraph *g, uint32_t n, uint32_t big_vertices, int cluster, uint32_t *order,
                    const unsigned long long *cost = nullptr);
