// Reverse CSR built on the device from the forward CSR (SCC_FLAG_DERIVE_REVERSE),
// and GTgraph text parsed into both CSRs on the device.
//
// The reference's loader builds both CSRs on the host from one arc list
// (load.cpp:47-113); the reverse one is a pure function of the forward one:
// in-lists in ascending source order, Br[0] = Br[1] = 0, Br[V+1] = E.  Here
// it is a stable sort of the forward arcs by destination: the forward CSR
// already lists the arcs by ascending source, so a stable sort leaves every
// in-list in ascending source order with no second sort.
//   1. expand: src[e] = the source of arc e, written 32 consecutive arcs
//      per warp step (offsets checked);
//   2. least-significant-digit radix sort of (Fc[e], src[e]) by Fc, 8 bits
//      a pass, as many passes as the vertex ids have bytes (3 for 2^22
//      vertices); each pass is a per-tile digit histogram, a scan of the
//      digit-major histogram matrix, and a scatter that ranks every tile's
//      arcs in shared memory (ballot multi-split + per-warp counters, stable), stages
//      them there in digit order and writes each digit's run contiguously;
//      the last pass writes the sources straight into Bc;
//   3. Br[v] = the first position whose key is >= v, one write per vertex
//      from the run boundaries of the sorted keys.
// No atomics on global memory: hub vertices with millions of in-arcs cost
// what any other vertex costs.  Ids outside [1, V] and malformed offsets set
// SCC_ERR_BAD_GRAPH in the control block, which stops the SCC kernel at its
// entry.  No counterpart in the reference (it builds both CSRs on the host).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/scc_b200.h"
#include "scc_internal.h"

using namespace sccb;

namespace {

constexpr uint32_t TILE = 8192;         // scan tile (1024 threads x 8)
constexpr uint32_t RS_T = 256;          // radix threads per CTA (one per digit)
constexpr uint32_t RS_W = RS_T / 32;    // warps per radix CTA
constexpr uint32_t RS_IPT = 16;         // arcs per thread
constexpr uint32_t RS_WARP_ITEMS = 32 * RS_IPT;
constexpr uint32_t RS_TILE = RS_T * RS_IPT;   // 4,096 arcs per radix tile
constexpr uint32_t RS_BINS = 256;
constexpr size_t RS_SMEM = (size_t)RS_TILE * 8;   // staged keys and values
constexpr uint32_t UP_CHUNKS = UPLOAD_CHUNKS;     // host-to-device pieces of the forward targets
constexpr uint32_t UP_MIN_TILES = 512;            // at least 2M arcs (8 MB) a piece

// Sum of every TILE-entry tile of in[0 .. n).
__global__ void __launch_bounds__(1024) k_tile_sums(const uint32_t *__restrict__ in, uint32_t n,
                                                    uint32_t *__restrict__ sums)
{
    __shared__ uint32_t s_w[32];
    const uint32_t base = blockIdx.x * TILE;
    uint32_t x = 0;
    for (uint32_t i = threadIdx.x; i < TILE; i += 1024u)
        if (base + i < n) x += in[base + i];
    x = __reduce_add_sync(0xFFFFFFFFu, x);
    if ((threadIdx.x & 31u) == 0u) s_w[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32u) {
        const uint32_t y = __reduce_add_sync(0xFFFFFFFFu, s_w[threadIdx.x]);
        if (threadIdx.x == 0) sums[blockIdx.x] = y;
    }
}

// Block-wide exclusive scan of one value per thread (1024 threads); *total
// receives the sum.
__device__ __forceinline__ uint32_t block_scan1024(uint32_t x, uint32_t *total)
{
    __shared__ uint32_t s_w[32];
    const uint32_t lane = threadIdx.x & 31u, wi = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31u) s_w[wi] = incl;
    __syncthreads();
    if (wi == 0) {
        const uint32_t w = s_w[lane];
        uint32_t wincl = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wincl, o);
            if (lane >= (uint32_t)o) wincl += y;
        }
        s_w[lane] = wincl - w;
        if (lane == 31u) *total = wincl;
    }
    __syncthreads();
    const uint32_t r = s_w[wi] + incl - x;
    __syncthreads();
    return r;
}

// Exclusive scan of the tile sums in place (one CTA); sums[ntiles] receives
// the total.
__global__ void __launch_bounds__(1024) k_scan_sums(uint32_t *sums, uint32_t ntiles)
{
    __shared__ uint32_t s_tot;
    uint32_t run = 0;
    for (uint32_t base = 0; base < ntiles; base += 1024u) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t x = i < ntiles ? sums[i] : 0u;
        const uint32_t ex = block_scan1024(x, &s_tot);
        if (i < ntiles) sums[i] = run + ex;
        __syncthreads();
        run += s_tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[ntiles] = run;
}

// out = exclusive prefix of in[0 .. n), given the scanned tile sums.
__global__ void __launch_bounds__(1024) k_tile_scan(const uint32_t *__restrict__ in, uint32_t n,
                                                    const uint32_t *__restrict__ sums, uint32_t *__restrict__ out)
{
    __shared__ uint32_t s_tot;
    const uint32_t base = blockIdx.x * TILE + threadIdx.x * 8u;
    uint32_t x[8], s = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        x[j] = base + (uint32_t)j < n ? in[base + j] : 0u;
        s += x[j];
    }
    uint32_t run = sums[blockIdx.x] + block_scan1024(s, &s_tot);
#pragma unroll
    for (int j = 0; j < 8; j++) {
        if (base + (uint32_t)j < n) out[base + j] = run;
        run += x[j];
    }
}

// 1. src[e] = the source of arc e, one XA-arc tile per CTA: the sources
// owning the tile's arcs are the vertices from the owner of its first arc to
// the owner of the next tile's first arc (k_tr_tile_owner); each of them
// writes its arcs inside the tile into shared memory (runs longer than 32
// by the whole warp), then the tile goes out with coalesced stores.  Hubs
// cost what any tile costs.  Offsets are checked (the reference layout:
// Fr[0] = Fr[1] = 0, non-decreasing, Fr[V+1] = E); with malformed ones the
// window is clamped to [1, V] and every store stays inside the tile.
constexpr uint32_t XT = 256;            // expand threads per CTA
constexpr uint32_t XA = 4096;           // arcs per expand tile
constexpr uint32_t XW = 8;              // window offsets per thread and round

// own[c] = the source of arc c * XA: u owns the tile starts in [Fr[u], Fr[u+1]).
__global__ void k_tr_tile_owner(const uint32_t *__restrict__ Fr, uint32_t V, uint32_t E, uint32_t *__restrict__ own,
                                Ctl *ctl)
{
    if (blockIdx.x == 0 && threadIdx.x == 0 && (Fr[0] != 0u || Fr[1] != 0u || Fr[V + 1] != E))
        set_error(ctl, E_BAD_GRAPH, 70);
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x + 1u; u <= V; u += gridDim.x * blockDim.x) {
        const uint32_t b = Fr[u], e = Fr[u + 1];
        if (b > e || e > E) {
            set_error(ctl, E_BAD_GRAPH, 71);
            continue;
        }
        for (uint64_t c = ((uint64_t)b + XA - 1u) / XA; c * XA < e; c++) own[c] = u;
    }
}

__global__ void __launch_bounds__(XT) k_tr_expand(const uint32_t *__restrict__ Fr, uint32_t V, uint32_t E,
                                                  const uint32_t *__restrict__ own, uint32_t *__restrict__ src)
{
    __shared__ __align__(16) uint32_t s_src[XA];
    __shared__ uint32_t s_w[XT / 32];
    const uint32_t lane = threadIdx.x & 31u, wi = threadIdx.x >> 5;
    const uint32_t ntiles = (uint32_t)(((uint64_t)E + XA - 1u) / XA);
    for (uint32_t c = blockIdx.x; c < ntiles; c += gridDim.x) {
        const uint32_t t0 = c * XA, m = min(XA, E - t0);
        const uint32_t lo = min(max(own[c], 1u), V);
        const uint32_t hi = c + 1u < ntiles ? min(max(own[c + 1], lo), V) : V;
        for (uint32_t i = threadIdx.x; i < XA; i += XT) s_src[i] = 0u;
        __syncthreads();
        // every source with arcs in the tile marks the first of them
        for (uint32_t u0 = lo; u0 <= hi; u0 += XT * XW) {
            uint32_t ob[XW + 1];
#pragma unroll
            for (uint32_t q = 0; q <= XW; q++) {
                const uint32_t u = u0 + threadIdx.x * XW + q;
                ob[q] = u <= hi + 1u ? Fr[u] : 0u;
            }
#pragma unroll
            for (uint32_t q = 0; q < XW; q++) {
                const uint32_t u = u0 + threadIdx.x * XW + q;
                const uint32_t a = max(ob[q], t0);
                if (u <= hi && a < min(ob[q + 1], t0 + m)) s_src[a - t0] = u;
            }
        }
        __syncthreads();
        // arc i's source = the last mark at or before i (sources increase along the tile)
        uint32_t x[XA / XT];
#pragma unroll
        for (uint32_t q = 0; q < XA / XT; q += 4) {
            const uint4 y = *reinterpret_cast<const uint4 *>(&s_src[threadIdx.x * (XA / XT) + q]);
            x[q] = y.x; x[q + 1] = y.y; x[q + 2] = y.z; x[q + 3] = y.w;
        }
        uint32_t run = 0;
#pragma unroll
        for (uint32_t q = 0; q < XA / XT; q++) x[q] = run = max(run, x[q]);
        uint32_t incl = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= (uint32_t)o) incl = max(incl, y);
        }
        if (lane == 31u) s_w[wi] = incl;
        __syncthreads();
        uint32_t excl = __shfl_up_sync(0xFFFFFFFFu, incl, 1);
        if (lane == 0u) excl = 0u;
        for (uint32_t q = 0; q < wi; q++) excl = max(excl, s_w[q]);
        const uint32_t i0 = threadIdx.x * (XA / XT);
        if (i0 + XA / XT <= m) {
#pragma unroll
            for (uint32_t q = 0; q < XA / XT; q += 4)
                *reinterpret_cast<uint4 *>(&src[t0 + i0 + q]) =
                    make_uint4(max(x[q], excl), max(x[q + 1], excl), max(x[q + 2], excl), max(x[q + 3], excl));
        } else {
#pragma unroll
            for (uint32_t q = 0; q < XA / XT; q++)
                if (i0 + q < m) src[t0 + i0 + q] = max(x[q], excl);
        }
        __syncthreads();
    }
}

// Digits of one radix tile; warp w holds arcs [w*512, w*512+512) of the
// tile, lane l its arcs l, l+32, ...
// (n < 2^32, so slot numbers fit 32 bits.)
__device__ __forceinline__ uint32_t rs_slot(uint32_t tile, uint32_t j)
{
    return tile * RS_TILE + (threadIdx.x >> 5) * RS_WARP_ITEMS + j * 32u + (threadIdx.x & 31u);
}

// Lanes of the warp whose 8-bit digit equals this lane's (warp multi-split
// by ballots); valid lanes only.
__device__ __forceinline__ uint32_t rs_peers(uint32_t d, bool valid)
{
    uint32_t m = __ballot_sync(0xFFFFFFFFu, valid);
#pragma unroll
    for (uint32_t b = 0; b < 8u; b++) {
        const uint32_t bit = (d >> b) & 1u;
        m &= ~(__ballot_sync(0xFFFFFFFFu, bit) ^ (0u - bit));   // lanes whose bit b equals ours
    }
    return m;
}

// Rank of every arc of this warp's slice among the slice's arcs with the
// same digit (arcs taken in slice order: j, then lane); arcs j < nv of the
// thread exist.  cw holds the warp's running count per digit: the lowest
// lane of each digit group adds the group's size and shares the old count
// (one warp's shared-memory atomics complete in instruction order, so the
// counts follow j).
__device__ __forceinline__ void rs_rank(const uint32_t (&k)[RS_IPT], uint32_t nv, uint32_t shift, uint32_t dm,
                                        uint32_t (&rank)[RS_IPT], uint32_t *cw)
{
    uint32_t lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
#pragma unroll
    for (int j = 0; j < (int)RS_IPT; j++) {
        const bool valid = (uint32_t)j < nv;
        const uint32_t d = (k[j] >> shift) & dm;
        const uint32_t peers = rs_peers(d, valid);
        const uint32_t lead = __ffs(peers) - 1u;
        uint32_t before = 0;
        if (valid && (peers & lt) == 0u) before = atomicAdd(&cw[d], (uint32_t)__popc(peers));
        before = __shfl_sync(0xFFFFFFFFu, before, lead & 31u);
        rank[j] = before + __popc(peers & lt);
    }
}

// Arcs of this thread inside a tile of n arcs (slots j < the result).
__device__ __forceinline__ uint32_t rs_valid(uint32_t tile, uint32_t n)
{
    const uint32_t b = rs_slot(tile, 0);
    const uint32_t q = b >= n ? 0u : (n - b - 1u) / 32u + 1u;
    return q < RS_IPT ? q : RS_IPT;
}

// 2a. per-tile digit counts, digit-major: H[d * ntiles + tile], for tiles
// tile0 + blockIdx.x; a digit is key bits [shift, shift + nb).  With ctl,
// keys outside [1, V] are flagged.
__global__ void __launch_bounds__(RS_T) k_rs_hist(const uint32_t *__restrict__ keys, uint32_t n, uint32_t shift,
                                                  uint32_t nb, uint32_t ntiles, uint32_t tile0,
                                                  uint32_t *__restrict__ H, uint32_t V, Ctl *ctl)
{
    const uint32_t tile = tile0 + blockIdx.x;
    const uint32_t dm = (1u << nb) - 1u;
    __shared__ uint32_t cnt[RS_W][RS_BINS];
    for (uint32_t i = threadIdx.x; i < RS_W * RS_BINS; i += RS_T) (&cnt[0][0])[i] = 0u;
    __syncthreads();
    uint32_t k[RS_IPT];
    bool bad = false;
#pragma unroll
    for (int j = 0; j < (int)RS_IPT; j++) {
        const uint32_t i = rs_slot(tile, j);
        k[j] = i < n ? __ldg(&keys[i]) : 0u;
    }
    uint32_t *cw = cnt[threadIdx.x >> 5];
#pragma unroll
    for (int j = 0; j < (int)RS_IPT; j++)
        if (rs_slot(tile, j) < n) {
            bad |= k[j] - 1u >= V;
            atomicAdd(&cw[(k[j] >> shift) & dm], 1u);
        }
    if (ctl && bad) set_error(ctl, E_BAD_GRAPH, 72);
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < RS_BINS; b += RS_T) {
        uint32_t s = 0;
#pragma unroll
        for (uint32_t w = 0; w < RS_W; w++) s += cnt[w][b];
        H[(size_t)b * ntiles + tile] = s;
    }
}

// 2b. stable scatter of one tile by its digit: Hs = exclusive scan of H
// (digit-major), so Hs[d * ntiles + tile] is where the tile's run of digit
// d starts in the output.  Keys stay in registers through the ranking, the
// values are read when the tile is staged; four CTAs per SM overlap one
// tile's loads with another's ranking.
__global__ void __launch_bounds__(RS_T, 4) k_rs_scatter(const uint32_t *__restrict__ kin,
                                                        const uint32_t *__restrict__ vin, uint32_t *__restrict__ kout,
                                                        uint32_t *__restrict__ vout, uint32_t n, uint32_t shift,
                                                        uint32_t nb, uint32_t ntiles, const uint32_t *__restrict__ Hs)
{
    extern __shared__ uint32_t s_stage[];   // RS_TILE staged keys, then RS_TILE staged values
    __shared__ uint32_t cnt[RS_W][RS_BINS];
    __shared__ uint32_t s_loc[RS_BINS], s_glob[RS_BINS], s_wsum[RS_BINS / 32];
    const uint32_t dm = (1u << nb) - 1u;
    uint32_t *sk = s_stage, *sv = s_stage + RS_TILE;
    if (threadIdx.x < RS_BINS) s_glob[threadIdx.x] = Hs[(size_t)threadIdx.x * ntiles + blockIdx.x];
    for (uint32_t i = threadIdx.x; i < RS_W * RS_BINS; i += RS_T) (&cnt[0][0])[i] = 0u;
    uint32_t k[RS_IPT], r[RS_IPT];
    const uint32_t nv = rs_valid(blockIdx.x, n);
#pragma unroll
    for (int j = 0; j < (int)RS_IPT; j++) k[j] = (uint32_t)j < nv ? __ldg(&kin[rs_slot(blockIdx.x, j)]) : 0u;
    __syncthreads();
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    rs_rank(k, nv, shift, dm, r, cnt[w]);
    __syncthreads();
    // per digit: exclusive prefix over the warps, the tile's total, its start
    uint32_t tot = 0;
    if (threadIdx.x < RS_BINS) {
        const uint32_t b = threadIdx.x;
#pragma unroll
        for (uint32_t q = 0; q < RS_W; q++) {
            const uint32_t c = cnt[q][b];
            cnt[q][b] = tot;
            tot += c;
        }
        uint32_t incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= (uint32_t)o) incl += y;
        }
        if (lane == 31u) s_wsum[w] = incl;
        s_loc[b] = incl - tot;
    }
    __syncthreads();
    if (threadIdx.x < RS_BINS) {
        uint32_t add = 0;
        for (uint32_t q = 0; q < w; q++) add += s_wsum[q];
        s_loc[threadIdx.x] += add;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < (int)RS_IPT; j++)
        if ((uint32_t)j < nv) {
            const uint32_t d = (k[j] >> shift) & dm;
            const uint32_t p = s_loc[d] + cnt[w][d] + r[j];
            sk[p] = k[j];
            sv[p] = __ldg(&vin[rs_slot(blockIdx.x, j)]);
        }
    __syncthreads();
    const uint32_t t0 = blockIdx.x * RS_TILE, m = min(RS_TILE, n - t0);
    for (uint32_t i = threadIdx.x; i < m; i += RS_T) {
        const uint32_t key = sk[i], dg = (key >> shift) & dm;
        const uint32_t pos = s_glob[dg] + (i - s_loc[dg]);
        kout[pos] = key;
        vout[pos] = sv[i];
    }
}

// 3. R[v] = number of keys below v for v in [0, V+1] from the sorted keys
// K[0 .. n): position i owns the vertices (K[i-1], K[i]] (K[-1] = 0,
// K[n] = V+1; keys clamped to V+1).  Eight positions per thread (two 16-byte
// loads); gaps longer than 32 vertices are written by the whole warp.
__global__ void k_tr_offsets(const uint32_t *__restrict__ K, uint32_t n, uint32_t V, uint32_t *__restrict__ R)
{
    const uint32_t lane = threadIdx.x & 31u;
    if (blockIdx.x == 0 && threadIdx.x == 0) R[0] = 0u;
    const uint64_t nt = ((uint64_t)n + 1u + 7u) / 8u;   // threads' worth of positions 0 .. n
    for (uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x; t0 < nt; t0 += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t t = t0 + threadIdx.x, i0 = t * 8u;
        uint32_t key[9];
#pragma unroll
        for (int j = 0; j < 9; j++) key[j] = V + 1u;
        if (t < nt) {
            key[0] = i0 ? K[i0 - 1u] : 0u;
            if (i0 + 8u <= n) {
                const uint4 x = *reinterpret_cast<const uint4 *>(K + i0);
                const uint4 y = *reinterpret_cast<const uint4 *>(K + i0 + 4u);
                key[1] = x.x; key[2] = x.y; key[3] = x.z; key[4] = x.w;
                key[5] = y.x; key[6] = y.y; key[7] = y.z; key[8] = y.w;
            } else {
#pragma unroll
                for (int j = 0; j < 8; j++)
                    if (i0 + j < n) key[1 + j] = K[i0 + j];
            }
        }
        key[0] = min(key[0], V + 1u);
#pragma unroll
        for (int j = 1; j < 9; j++) key[j] = max(min(key[j], V + 1u), key[j - 1]);
        // positions past n own nothing (their keys are V + 1); the usual case,
        // every gap of the thread short, is written by the thread alone
        const bool longgap = key[8] - key[0] > 32u;
        if (!longgap) {
#pragma unroll
            for (int j = 0; j < 8; j++)
                for (uint32_t x = key[j] + 1u; x <= key[j + 1]; x++) R[x] = (uint32_t)(i0 + j);
        }
        if (__ballot_sync(0xFFFFFFFFu, longgap)) {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const uint32_t a = longgap ? key[j] : 0u, b = longgap ? key[j + 1] : 0u;
                if (b - a <= 32u)
                    for (uint32_t x = a + 1u; x <= b; x++) R[x] = (uint32_t)(i0 + j);
                unsigned hm = __ballot_sync(0xFFFFFFFFu, b - a > 32u);
                while (hm) {
                    const unsigned q = __ffs(hm) - 1u;
                    hm &= hm - 1u;
                    const uint32_t aq = __shfl_sync(0xFFFFFFFFu, a, q), bq = __shfl_sync(0xFFFFFFFFu, b, q);
                    const uint32_t iq = (uint32_t)__shfl_sync(0xFFFFFFFFu, (uint32_t)(i0 + j), q);
                    for (uint32_t x = aq + 1u + lane; x <= bq; x += 32u) R[x] = iq;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------
// GTgraph text parsed on the device (load.cpp:32-77).  The host reads the
// file and its header (7 lines, then "p sp V E"); the rest -- one arc
// "a u v w" per line -- is copied to the device and every thread takes
// the lines that start in its 64-byte segment, the lanes of a warp one
// line each per step (so their parses run side by side): one pass counts
// the records (non-blank lines) of every segment, a scan gives each
// segment its first record index, the second pass parses and writes record
// r's (u, v).  Two stable radix sorts (by v, then by u) then order the arcs
// by (u, v) as the reference's std::sort does (load.cpp:47), duplicates and
// self-loops kept, and the reverse CSR is derived from the forward one.
// ---------------------------------------------------------------------
constexpr uint32_t SEG = 64;            // bytes of text per thread
constexpr uint32_t PT = 256;            // threads per parse CTA

__device__ __forceinline__ bool tws(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// The first line that starts in [b, e) (a line starts at 0 and after every
// '\n'), or e.
__device__ __forceinline__ uint64_t first_line(const char *T, uint64_t b, uint64_t e)
{
    if (b == 0) return 0;
    uint64_t p = b;
    while (p < e && T[p - 1] != '\n') p++;
    return p;
}

// Past the '\n' that ends the line p is in (or L).
__device__ __forceinline__ uint64_t line_end(const char *T, uint64_t p, uint64_t L)
{
    while (p < L && T[p] != '\n') p++;
    return p < L ? p + 1 : L;
}

// Parses the line starting at p and moves p past it: 0 blank, 1 an arc
// (u, v), -1 malformed.
__device__ int parse_line(const char *T, uint64_t &p, uint64_t L, uint32_t V, uint32_t &u, uint32_t &v)
{
    int kind = 1;
    while (p < L && tws(T[p])) p++;
    if (p >= L || T[p] == '\n') {
        kind = 0;
    } else {
        p++;   // the arc letter (one character, as the reference reads it, load.cpp:43)
        uint64_t x[3] = {0, 0, 0};
        for (int k = 0; k < 3 && kind > 0; k++) {
            while (p < L && tws(T[p])) p++;
            if (p >= L || T[p] < '0' || T[p] > '9') {
                kind = -1;
                break;
            }
            uint64_t y = 0;
            while (p < L && T[p] >= '0' && T[p] <= '9' && y <= 0xFFFFFFFFull) y = y * 10u + (uint64_t)(T[p++] - '0');
            if (y > 0xFFFFFFFFull) kind = -1;
            x[k] = y;
        }
        if (kind > 0) {
            while (p < L && tws(T[p])) p++;
            if ((p < L && T[p] != '\n') || x[0] < 1u || x[0] > V || x[1] < 1u || x[1] > V) kind = -1;
            u = (uint32_t)x[0];
            v = (uint32_t)x[1];
        }
    }
    p = line_end(T, p, L);
    return kind;
}

// Records (non-blank lines) that start in thread t's segment.  Every lane
// walks its own lines, all lanes of a warp one line per step.
__device__ uint32_t seg_records(const char *T, uint64_t L, uint64_t t)
{
    const uint64_t b = t * SEG, e = min(b + SEG, L);
    uint32_t n = 0;
    for (uint64_t p = first_line(T, b, e); p < e;) {
        while (p < L && tws(T[p])) p++;
        if (p < L && T[p] != '\n') n++;
        p = line_end(T, p, L);
    }
    return n;
}

__device__ __forceinline__ uint32_t block_excl256(uint32_t x, uint32_t *total)
{
    __shared__ uint32_t s_w[PT / 32];
    const uint32_t lane = threadIdx.x & 31u, wi = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31u) s_w[wi] = incl;
    __syncthreads();
    uint32_t before = 0, all = 0;
    for (uint32_t i = 0; i < PT / 32; i++) {
        if (i < wi) before += s_w[i];
        all += s_w[i];
    }
    *total = all;
    __syncthreads();
    return before + incl - x;
}

__global__ void __launch_bounds__(PT) k_parse_count(const char *T, uint64_t L, uint32_t *sums)
{
    uint32_t tot;
    const uint32_t n = seg_records(T, L, (uint64_t)blockIdx.x * PT + threadIdx.x);
    block_excl256(n, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Second pass: record r of the file goes to src[r], dst[r] (r < E); lines
// that do not parse as an arc raise SCC_ERR_BAD_GRAPH.  sums: exclusive
// scan of the per-CTA counts.
__global__ void __launch_bounds__(PT) k_parse_write(const char *T, uint64_t L, uint32_t V, uint32_t E,
                                                    const uint32_t *sums, uint32_t *src, uint32_t *dst, Ctl *ctl)
{
    uint32_t tot;
    const uint64_t t = (uint64_t)blockIdx.x * PT + threadIdx.x;
    uint32_t r = sums[blockIdx.x] + block_excl256(seg_records(T, L, t), &tot);
    const uint64_t b = t * SEG, e = min(b + SEG, L);
    for (uint64_t p = first_line(T, b, e); p < e;) {
        uint32_t u = 0, v = 0;
        const int k = parse_line(T, p, L, V, u, v);
        if (k < 0) {
            if (r < E) set_error(ctl, E_BAD_GRAPH, 74);   // the reference stops reading after E arcs (load.cpp:42)
            r++;
        } else if (k > 0) {
            if (r < E) { src[r] = u; dst[r] = v; }
            r++;
        }
    }
}

}  // namespace

namespace {

// Temporaries of the sorts (kept in the context): three arc-sized arrays,
// the digit histogram matrix and its scan, the scan's tile sums.
struct TrBufs {
    uint32_t *t[3];
    uint32_t *H, *Hs, *sums;
};

int tr_prepare(scc_context *ctx, uint64_t E, size_t extra_sums, TrBufs *b)
{
    const size_t ne = std::max<size_t>(E, 1);
    const size_t nh = (size_t)RS_BINS * ((ne + RS_TILE - 1) / RS_TILE);
    const size_t nsum = std::max<size_t>((nh + TILE - 1) / TILE, extra_sums) + 64;
    const size_t tmp_bytes = (2 * nh + nsum) * 4;
    if (ne > ctx->tcapE || tmp_bytes > ctx->ttmp_bytes) {
        for (auto &p : ctx->tarc) { cudaFree(p); p = nullptr; }
        cudaFree(ctx->ttmp);
        ctx->ttmp = nullptr;
        ctx->tcapE = 0;
        ctx->ttmp_bytes = 0;
        for (auto &p : ctx->tarc)
            if (cudaMalloc((void **)&p, ne * 4) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_OOM; }
        if (cudaMalloc(&ctx->ttmp, tmp_bytes) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_OOM; }
        ctx->tcapE = ne;
        ctx->ttmp_bytes = tmp_bytes;
    }
    if (cudaFuncSetAttribute(k_rs_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS_SMEM) != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    for (int i = 0; i < 3; i++) b->t[i] = ctx->tarc[i];
    b->H = (uint32_t *)ctx->ttmp;
    b->Hs = b->H + nh;
    b->sums = b->Hs + nh;
    return SCC_OK;
}

// Bits of a vertex id in [1, V].
uint32_t id_bits(uint32_t V) { return V ? (uint32_t)(32 - __builtin_clz(V)) : 0u; }

// Digit bits of the pass at shift (fewer above the ids' top bit).
uint32_t pass_bits(uint32_t V, uint32_t shift) { return std::min(8u, id_bits(V) - shift); }

// One stable pass: (kin, vin) -> (kout, vout) ordered by key bits
// [shift, shift + 8).  With ctl, keys outside [1, V] are flagged.  With
// hist false the caller has already counted the tiles' digits into b.H.
void rs_pass(const TrBufs &b, uint32_t n, uint32_t shift, const uint32_t *kin, const uint32_t *vin, uint32_t *kout,
             uint32_t *vout, uint32_t V, Ctl *ctl, cudaStream_t st, bool hist = true)
{
    const uint32_t nt = (n + RS_TILE - 1) / RS_TILE, nh = nt * RS_BINS, ht = (nh + TILE - 1) / TILE;
    const uint32_t nb = pass_bits(V, shift);
    if (hist) k_rs_hist<<<nt, RS_T, 0, st>>>(kin, n, shift, nb, nt, 0u, b.H, V, ctl);
    k_tile_sums<<<ht, 1024, 0, st>>>(b.H, nh, b.sums);
    k_scan_sums<<<1, 1024, 0, st>>>(b.sums, ht);
    k_tile_scan<<<ht, 1024, 0, st>>>(b.H, nh, b.sums, b.Hs);
    k_rs_scatter<<<nt, RS_T, RS_SMEM, st>>>(kin, vin, kout, vout, n, shift, nb, nt, b.Hs);
}

// The upload stream of the context (created on first use) and its events.
int upload_stream(scc_context *ctx)
{
    if (!ctx->up && cudaStreamCreateWithFlags(&ctx->up, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    for (auto &e : ctx->upev)
        if (!e && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return SCC_ERR_CUDA;
        }
    return SCC_OK;
}

// Radix passes a vertex id in [1, V] needs.
uint32_t id_passes(uint32_t V) { return (id_bits(V) + 7u) / 8u; }

int launched() { return cudaGetLastError() == cudaSuccess ? SCC_OK : SCC_ERR_CUDA; }

}  // namespace

int sccb_derive_reverse(scc_context *ctx, const uint32_t *dFr, const uint32_t *dFc, uint32_t V, uint32_t E,
                        uint32_t *dBr, uint32_t *dBc, Ctl *ctl, cudaStream_t st, const uint32_t *hFc)
{
    TrBufs b;
    int rc = tr_prepare(ctx, E, 0, &b);
    if (rc != SCC_OK) return rc;
    const uint32_t P = E ? id_passes(V) : 0u;
    // With hFc the forward targets are still in host memory: they cross in
    // chunks on the context's upload stream while the expand (which needs
    // Fr only) runs, and each chunk's tiles are counted as soon as it lands.
    const uint32_t nt = (E + RS_TILE - 1) / RS_TILE;
    uint32_t nchunks = 0, chunk_tiles = 0;
    if (hFc && P) {
        if ((rc = upload_stream(ctx)) != SCC_OK) return rc;
        chunk_tiles = std::max((nt + UP_CHUNKS - 1) / UP_CHUNKS, UP_MIN_TILES);
        nchunks = (nt + chunk_tiles - 1) / chunk_tiles;
        if (cudaEventRecord(ctx->upev[UP_CHUNKS], st) != cudaSuccess ||   // earlier work on st is done with dFc
            cudaStreamWaitEvent(ctx->up, ctx->upev[UP_CHUNKS], 0) != cudaSuccess) {
            cudaGetLastError();
            return SCC_ERR_CUDA;
        }
        for (uint32_t c = 0; c < nchunks; c++) {
            const size_t a0 = (size_t)c * chunk_tiles * RS_TILE, a1 = std::min<size_t>(a0 + (size_t)chunk_tiles * RS_TILE, E);
            if (cudaMemcpyAsync(const_cast<uint32_t *>(dFc) + a0, hFc + a0, (a1 - a0) * 4, cudaMemcpyHostToDevice,
                                ctx->up) != cudaSuccess ||
                cudaEventRecord(ctx->upev[c], ctx->up) != cudaSuccess) {
                cudaGetLastError();
                return SCC_ERR_CUDA;
            }
        }
    } else if (hFc && E) {
        if (cudaMemcpyAsync(const_cast<uint32_t *>(dFc), hFc, (size_t)E * 4, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            cudaGetLastError();
            return SCC_ERR_CUDA;
        }
    }
    // the sources ping-pong between t[2] and Bc so that the last pass writes Bc
    uint32_t *vin = (P & 1u) ? b.t[2] : dBc;
    uint32_t *own = b.t[0];   // tile owners, read by the expand before pass 0 writes keys there
    k_tr_tile_owner<<<ctx->nsm * 8, 256, 0, st>>>(dFr, V, E, own, ctl);
    if (E) k_tr_expand<<<ctx->nsm * 8, XT, 0, st>>>(dFr, V, E, own, vin);
    for (uint32_t c = 0; c < nchunks; c++) {
        const uint32_t t0 = c * chunk_tiles, tn = std::min(chunk_tiles, nt - t0);
        if (cudaStreamWaitEvent(st, ctx->upev[c], 0) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_CUDA; }
        k_rs_hist<<<tn, RS_T, 0, st>>>(dFc, E, 0u, pass_bits(V, 0u), nt, t0, b.H, V, ctl);
    }
    const uint32_t *kin = dFc;
    for (uint32_t p = 0; p < P; p++) {
        uint32_t *kout = b.t[p & 1u], *vout = vin == b.t[2] ? dBc : b.t[2];
        rs_pass(b, E, 8u * p, kin, vin, kout, vout, V, p == 0 ? ctl : nullptr, st, !(p == 0 && nchunks));
        kin = kout;
        vin = vout;
    }
    k_tr_offsets<<<ctx->nsm * 8, 256, 0, st>>>(kin, P ? E : 0u, V, dBr);
    return launched();
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
    int rc = sccb_derive_reverse(ctx, Fr, Fc, V, E, Br, Bc, ctx->tctl, st, nullptr);
    if (rc != SCC_OK) return rc;
    int err = 0;
    if (cudaMemcpyAsync(&err, &ctx->tctl->error, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    return err ? err : SCC_OK;
}

// GTgraph text (or the binary CSR format) -> both CSRs in the context's
// device arrays; see include/scc_b200.h.
namespace {

constexpr size_t STAGE = 64u << 20;     // bytes of one page-locked staging buffer
constexpr size_t HEAD = 1u << 20;       // the text header must end within this many bytes

struct File {
    FILE *f = nullptr;
    ~File() { if (f) fclose(f); }
};

int stage_buffers(scc_context *ctx)
{
    for (int i = 0; i < 2; i++) {
        if (!ctx->hstage[i] && cudaHostAlloc((void **)&ctx->hstage[i], STAGE, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return SCC_ERR_OOM;
        }
        if (!ctx->stage_ev[i] && cudaEventCreateWithFlags(&ctx->stage_ev[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return SCC_ERR_CUDA;
        }
    }
    return SCC_OK;
}

// Bytes [off, off + len) of the file to dst (device) through the two
// page-locked staging buffers: reading a piece overlaps the copy of the one
// before.  k counts pieces across calls (which buffer is next).
int stream_file(scc_context *ctx, FILE *f, uint64_t off, uint64_t len, char *dst, cudaStream_t st, unsigned &k)
{
    if (len && fseeko(f, (off_t)off, SEEK_SET) != 0) return SCC_ERR_IO;
    for (uint64_t done = 0; done < len;) {
        const size_t n = (size_t)std::min<uint64_t>(STAGE, len - done);
        const unsigned i = k++ & 1u;
        if (cudaEventSynchronize(ctx->stage_ev[i]) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_CUDA; }
        if (fread(ctx->hstage[i], 1, n, f) != n) return SCC_ERR_IO;
        if (cudaMemcpyAsync(dst + done, ctx->hstage[i], n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaEventRecord(ctx->stage_ev[i], st) != cudaSuccess) {
            cudaGetLastError();
            return SCC_ERR_CUDA;
        }
        done += n;
    }
    return SCC_OK;
}

}  // namespace

// GTgraph text (or the binary CSR format) -> both CSRs in the context's
// device arrays; see include/scc_b200.h.
extern "C" int scc_load_graph_device(scc_context *ctx, const char *path, scc_csr_view *out, void *stream)
{
    if (!ctx || !path || !out) return SCC_ERR_INVALID_ARG;
    memset(out, 0, sizeof(*out));
    File file;
    file.f = fopen(path, "rb");
    if (!file.f || fseeko(file.f, 0, SEEK_END) != 0) return SCC_ERR_IO;
    const off_t fsize = ftello(file.f);
    if (fsize <= 0 || fseeko(file.f, 0, SEEK_SET) != 0) return SCC_ERR_IO;
    const uint64_t size = (uint64_t)fsize;
    std::vector<char> hb((size_t)std::min<uint64_t>(size, HEAD));
    if (fread(hb.data(), 1, hb.size(), file.f) != hb.size()) return SCC_ERR_IO;
    const char *s = hb.data(), *e = s + hb.size();
    uint64_t V = 0, E = 0, body_off = 0;
    const bool bin = size >= 24 && memcmp(s, "SCCBIN01", 8) == 0;
    if (bin) {
        memcpy(&V, s + 8, 8);
        memcpy(&E, s + 16, 8);
        if (V > SCC_MAX_VERTICES || E > SCC_MAX_EDGES) return SCC_ERR_TOO_LARGE;
        if (size != 24 + 4 * (2 * (V + 2) + 2 * E)) return SCC_ERR_BAD_GRAPH;
    } else {
        // load.cpp:32-36: seven header lines, then "p sp V E"
        for (int i = 0; i < 7; i++) {
            while (s < e && *s != '\n') s++;
            if (s < e) s++;
        }
        auto ws = [&](const char *q) { while (q < e && (*q == ' ' || *q == '\t' || *q == '\n' || *q == '\r')) q++; return q; };
        auto tok = [&](const char *q) { while (q < e && !(*q == ' ' || *q == '\t' || *q == '\n' || *q == '\r')) q++; return q; };
        auto num = [&](const char *&q, uint64_t &x) {
            q = ws(q);
            if (q >= e || *q < '0' || *q > '9') return false;
            x = 0;
            while (q < e && *q >= '0' && *q <= '9') x = x * 10 + (uint64_t)(*q++ - '0');
            return q < e || hb.size() == size;   // a number cut by the end of the header window is not read
        };
        s = tok(ws(s));
        s = tok(ws(s));
        if (!num(s, V) || !num(s, E)) return SCC_ERR_BAD_GRAPH;
        if (V > SCC_MAX_VERTICES || E > SCC_MAX_EDGES) return SCC_ERR_TOO_LARGE;
        body_off = (uint64_t)(s - hb.data());
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (cudaSetDevice(ctx->device) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_NO_DEVICE; }
    cudaStream_t st = (cudaStream_t)stream;
    int rc = sccb_csr_mirror(ctx, (uint32_t)V, (uint32_t)E);
    if (rc != SCC_OK) return rc;
    if (!ctx->tctl && cudaMalloc((void **)&ctx->tctl, sizeof(Ctl)) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_OOM; }
    if (cudaMemsetAsync(ctx->tctl, 0, sizeof(Ctl), st) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_CUDA; }
    const size_t nv = (size_t)(V + 2) * 4, ne = (size_t)E * 4;
    if ((rc = stage_buffers(ctx)) != SCC_OK) return rc;
    unsigned piece = 0;
    if (bin) {
        if ((rc = stream_file(ctx, file.f, 24, nv, (char *)ctx->dFr, st, piece)) != SCC_OK ||
            (rc = stream_file(ctx, file.f, 24 + nv, ne, (char *)ctx->dFc, st, piece)) != SCC_OK ||
            (rc = stream_file(ctx, file.f, 24 + nv + ne, nv, (char *)ctx->dBr, st, piece)) != SCC_OK ||
            (rc = stream_file(ctx, file.f, 24 + 2 * nv + ne, ne, (char *)ctx->dBc, st, piece)) != SCC_OK) {
            cudaStreamSynchronize(st);
            cudaGetLastError();
            return rc;
        }
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            return SCC_ERR_CUDA;
        }
    } else {
        const uint64_t L = size - body_off;
        const uint64_t nblocks = std::max<uint64_t>((L + (uint64_t)PT * SEG - 1) / ((uint64_t)PT * SEG), 1);
        if (nblocks > 0x7FFFFFFFull) return SCC_ERR_TOO_LARGE;
        if (L + 16 > ctx->text_cap) {
            cudaFree(ctx->dtext);
            ctx->dtext = nullptr;
            ctx->text_cap = 0;
            if (cudaMalloc((void **)&ctx->dtext, L + 16) != cudaSuccess) { cudaGetLastError(); return SCC_ERR_OOM; }
            ctx->text_cap = L + 16;
        }
        TrBufs b;
        rc = tr_prepare(ctx, E, (size_t)nblocks + 1, &b);
        if (rc != SCC_OK) return rc;
        uint32_t *src = ctx->dBc, *dst = b.t[2];   // arcs in file order
        uint32_t total = 0;
        if ((rc = stream_file(ctx, file.f, body_off, L, ctx->dtext, st, piece)) != SCC_OK) {
            cudaStreamSynchronize(st);
            cudaGetLastError();
            return rc;
        }
        k_parse_count<<<(unsigned)nblocks, PT, 0, st>>>(ctx->dtext, L, b.sums);
        k_scan_sums<<<1, 1024, 0, st>>>(b.sums, (uint32_t)nblocks);
        k_parse_write<<<(unsigned)nblocks, PT, 0, st>>>(ctx->dtext, L, (uint32_t)V, (uint32_t)E, b.sums, src, dst,
                                                       ctx->tctl);
        if (cudaMemcpyAsync(&total, b.sums + nblocks, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            return SCC_ERR_CUDA;
        }
        if (total < E) return SCC_ERR_BAD_GRAPH;   // fewer arcs than the header announces
        // stable sort by v (values u), then by u (values v): arcs ordered by
        // (u, v) as load.cpp:47 orders them; the v column lands in Fc
        const uint32_t P = E ? id_passes((uint32_t)V) : 0u;
        uint32_t *pool[4] = {b.t[0], b.t[1], b.t[2], ctx->dBc};
        uint32_t *kin = dst, *vin = src;
        for (uint32_t q = 0; q < 2 * P; q++) {
            if (q == P) std::swap(kin, vin);
            uint32_t *vout = ctx->dFc, *kout = nullptr;
            for (uint32_t *p : pool)
                if (p != kin && p != vin) {
                    if (q + 1 < 2 * P && vout == ctx->dFc) vout = p;
                    else if (!kout) kout = p;
                }
            rs_pass(b, (uint32_t)E, 8u * (q % P), kin, vin, kout, vout, (uint32_t)V, nullptr, st);
            kin = kout;
            vin = vout;
        }
        k_tr_offsets<<<ctx->nsm * 8, 256, 0, st>>>(kin, P ? (uint32_t)E : 0u, (uint32_t)V, ctx->dFr);
        if ((rc = launched()) != SCC_OK) return rc;
        rc = sccb_derive_reverse(ctx, ctx->dFr, ctx->dFc, (uint32_t)V, (uint32_t)E, ctx->dBr, ctx->dBc, ctx->tctl, st,
                                 nullptr);
        if (rc != SCC_OK) return rc;
    }
    int err = 0;
    if (cudaMemcpyAsync(&err, &ctx->tctl->error, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return SCC_ERR_CUDA;
    }
    if (err) return err;
    *out = scc_csr_view{(uint32_t)V, (uint32_t)E, ctx->dFr, ctx->dFc, ctx->dBr, ctx->dBc};
    return SCC_OK;
}
