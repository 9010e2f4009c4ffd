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
    unsigned *next;             // work counter, zero before the launch
    uint32_t qcap, bu_k;
    int t1, t2, lw;
    unsigned long long timeout_ns;
};

// Shared memory of the batch kernel for a CTA size and staging slice.
size_t sccb_batch_smem(int threads, uint32_t qcap);
// Resident CTAs of the batch kernel on a device with nsm SMs.
int sccb_batch_ctas(int threads, uint32_t qcap, int nsm, uint32_t *out);
// Launch of the batch kernel (the caller zeroes p.next first).
int sccb_batch_launch(const BatchParams &p, int threads, bool hong, uint32_t ncta, cudaStream_t st);
