// Reverse CSR built on the device from the forward CSR (SCC_FLAG_DERIVE_REVERSE).
//
// The reference's loader builds both CSRs on the host from one arc list
// (load.cpp:47-113); the reverse one is a pure function of the forward one:
// in-lists in ascending source order, Br[0] = Br[1] = 0, Br[V+1] = E.  With
// the flag, scc_run copies only Fr and Fc across PCIe and rebuilds Br and Bc
// here: every edge gets its source id (one pass over the forward lists), a
// stable radix sort by target keeps the sources of each in-list ascending,
// and the offsets come from the sorted targets.  Ids outside [1, V] and
// malformed offsets set SCC_ERR_BAD_GRAPH in the control block, which stops
// the SCC kernel at its entry.  No counterpart in the reference.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <mutex>

#include "../../include/scc_b200.h"
#include "scc_internal.h"

using namespace sccb;

namespace {

// src[e] = u for every e in [Fr[u], Fr[u+1]): 32 vertices per warp, short
// lists by their lane, lists longer than 32 by the whole warp.
__global__ void k_edge_sources(const uint32_t *__restrict__ Fr, uint32_t V, uint32_t E, uint32_t *__restrict__ src,
                               Ctl *ctl)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0 && (Fr[0] != 0u || Fr[1] != 0u || Fr[V + 1] != E))
        set_error(ctl, E_BAD_GRAPH, 70);
    for (uint32_t base = warp * 32u; base < V; base += nwarps * 32u) {
        const uint32_t u = base + 1u + lane;
        uint32_t b = 0, e = 0;
        if (u <= V) {
            b = Fr[u];
            e = Fr[u + 1];
            if (b > e || e > E) {
                set_error(ctl, E_BAD_GRAPH, 71);
                b = e = 0;
            }
        }
        if (e - b <= 32u)
            for (uint32_t i = b; i < e; i++) src[i] = u;
        unsigned hm = __ballot_sync(0xFFFFFFFFu, e - b > 32u);
        while (hm) {
            const unsigned j = __ffs(hm) - 1u;
            hm &= hm - 1u;
            const uint32_t bj = __shfl_sync(0xFFFFFFFFu, b, j), ej = __shfl_sync(0xFFFFFFFFu, e, j);
            const uint32_t uj = base + 1u + j;
            for (uint32_t i = bj + lane; i < ej; i += 32u) src[i] = uj;
        }
    }
}

// Br from the sorted targets: the in-list of w starts at the first edge whose
// target is >= w.  Every boundary e (key[e] != key[e-1]) writes the starts
// of the ids in (key[e-1], key[e]]; ids after the last key start at E.
__global__ void k_rev_offsets(const uint32_t *__restrict__ key, uint32_t V, uint32_t E, uint32_t *__restrict__ Br,
                              Ctl *ctl)
{
    // the sort looked at the bits of V only, so every key is checked here
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, n = gridDim.x * blockDim.x;
    if (tid == 0) Br[0] = 0u;
    for (uint32_t e = tid; e < E; e += n) {
        const uint32_t k = key[e], kp = e ? key[e - 1] : 0u;
        if (k < 1u || k > V) {
            set_error(ctl, E_BAD_GRAPH, 72);
            continue;
        }
        for (uint32_t w = kp + 1u; w <= k; w++) Br[w] = e;   // empty unless kp < k (kp <= V when k is valid)
    }
    const uint32_t last = E ? min(key[E - 1], V) : 0u;
    for (uint32_t w = last + 1u + tid; w <= V + 1u; w += n) Br[w] = E;
}

}  // namespace

int sccb_derive_reverse(scc_context *ctx, const uint32_t *dFr, const uint32_t *dFc, uint32_t V, uint32_t E,
                        uint32_t *dBr, uint32_t *dBc, Ctl *ctl, cudaStream_t st)
{
    if (E > 0x7FFFFFFFu) return SCC_ERR_TOO_LARGE;   // the sort takes an int count
    const size_t ne = std::max<size_t>(E, 1);
    int bits = 1;   // key bits the sort looks at: those of V (larger ids are caught afterwards)
    while (bits < 32 && (V >> bits) != 0u) bits++;
    size_t tmp = 0;
    if (cub::DeviceRadixSort::SortPairs(nullptr, tmp, dFc, ctx->tkey, ctx->tsrc, dBc, (int)E, 0, bits, st) !=
        cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    if (ne > ctx->tcapE || tmp > ctx->ttmp_bytes) {
        cudaFree(ctx->tkey); cudaFree(ctx->tsrc); cudaFree(ctx->ttmp);
        ctx->tkey = ctx->tsrc = nullptr; ctx->ttmp = nullptr; ctx->tcapE = 0; ctx->ttmp_bytes = 0;
        if (cudaMalloc((void **)&ctx->tkey, ne * 4) != cudaSuccess || cudaMalloc((void **)&ctx->tsrc, ne * 4) != cudaSuccess ||
            cudaMalloc(&ctx->ttmp, std::max<size_t>(tmp, 16)) != cudaSuccess) {
            cudaGetLastError();
            return SCC_ERR_OOM;
        }
        ctx->tcapE = ne;
        ctx->ttmp_bytes = std::max<size_t>(tmp, 16);
    }
    const int blocks = ctx->nsm * 8;
    k_edge_sources<<<blocks, 256, 0, st>>>(dFr, V, E, ctx->tsrc, ctl);
    size_t tb = ctx->ttmp_bytes;
    if (E && cub::DeviceRadixSort::SortPairs(ctx->ttmp, tb, dFc, ctx->tkey, ctx->tsrc, dBc, (int)E, 0, bits, st) !=
                 cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    k_rev_offsets<<<blocks, 256, 0, st>>>(ctx->tkey, V, E, dBr, ctl);
    if (cudaGetLastError() != cudaSuccess) return SCC_ERR_CUDA;
    return SCC_OK;
}

extern "C" int scc_derive_reverse(scc_context *ctx, const uint32_t *Fr, const uint32_t *Fc, uint32_t V, uint32_t E,
                                  uint32_t *Br, uint32_t *Bc, void *stream)
{
    if (!ctx || !Fr || !Br || (E && (!Fc || !Bc))) return SCC_ERR_INVALID_ARG;
    if (V > SCC_MAX_VERTICES) return SCC_ERR_TOO_LARGE;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (cudaSetDevice(ctx->device) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_NO_DEVICE; }
    cudaStream_t st = (cudaStream_t)stream;
    if (!ctx->tctl && cudaMalloc((void **)&ctx->tctl, sizeof(Ctl)) != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_OOM;
    }
    if (cudaMemsetAsync(ctx->tctl, 0, sizeof(Ctl), st) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_CUDA; }
    int rc = sccb_derive_reverse(ctx, Fr, Fc, V, E, Br, Bc, ctx->tctl, st);
    if (rc != SCC_OK) return rc;
    int err = 0;
    if (cudaMemcpyAsync(&err, &ctx->tctl->error, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    return err ? err : SCC_OK;
}
