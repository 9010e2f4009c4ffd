"""Seeded synthetic graphs for the five benchmark configurations.

No public dataset is used: every graph is generated from a seed, with the
shapes, sizes and structure the configurations name.  Generation runs in
PyTorch on the CPU or on a CUDA device (large graphs are generated on the
GPU); a graph is reproducible for a given (seed, device).  Vertex ids are
1-based as in the reference.

* ``planted_random``  1,024 vertices, 8,192 uniform arcs (self-loops and
                      duplicates kept, as a GTgraph random graph may hold
                      them) plus 16 planted directed cycles of length 4-32.
* ``rmat``            R-MAT (a, b, c, d) = (0.57, 0.19, 0.19, 0.05), scale s,
                      edge factor 16; self-loops and duplicates removed;
                      optionally with randomly permuted vertex ids.
* ``grid``            n x n grid, 4-neighbour pairs; each pair is
                      bidirectional with p = 0.7, else one random
                      orientation; plus 0.1% x (grid arcs) uniform random
                      long-range arcs (self-loops excluded).
* ``batch_mix``       graphs with V log-uniform in [64, 65536] and mean
                      out-degree uniform in [4, 16]; half Erdos-Renyi, half
                      planted-SCC chains (strongly connected blocks, each a
                      cycle plus chords, linked acyclically).
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np
import torch

from .api import Graph


def _gen(seed: int, device) -> torch.Generator:
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


# ----------------------------------------------------------------------
# CSR construction
# ----------------------------------------------------------------------
def csr_from_arcs_torch(V: int, src: torch.Tensor, dst: torch.Tensor):
    """Reference-layout CSR from 1-based arcs, on the arcs' device.

    Forward lists are sorted by (u, v) and reverse lists by (v, u), which
    is the order load.cpp:47-113 produces (duplicates stay adjacent).
    Returns int32 tensors (Fr, Fc, Br, Bc); Fr/Br have V+2 entries.
    """
    src = src.to(torch.int64)
    dst = dst.to(torch.int64)
    M = V + 1
    key = torch.sort(src * M + dst).values
    s = key // M
    d = key - s * M
    cnt = torch.bincount(s, minlength=V + 2)[: V + 2]
    Fr = torch.zeros(V + 2, dtype=torch.int64, device=src.device)
    Fr[1:] = torch.cumsum(cnt, 0)[: V + 1]
    key2 = torch.sort(d * M + s).values
    d2 = key2 // M
    s2 = key2 - d2 * M
    cnt2 = torch.bincount(d2, minlength=V + 2)[: V + 2]
    Br = torch.zeros(V + 2, dtype=torch.int64, device=src.device)
    Br[1:] = torch.cumsum(cnt2, 0)[: V + 1]
    return Fr.to(torch.int32), d.to(torch.int32), Br.to(torch.int32), s2.to(torch.int32)


def to_graph(V: int, src: torch.Tensor, dst: torch.Tensor, name: str = "") -> Graph:
    Fr, Fc, Br, Bc = csr_from_arcs_torch(V, src, dst)
    f = lambda t: t.cpu().numpy().astype(np.uint32)  # noqa: E731
    return Graph(V, int(Fc.shape[0]), f(Fr), f(Fc), f(Br), f(Bc), name)


def dedup(V: int, src: torch.Tensor, dst: torch.Tensor, drop_self: bool = True):
    if drop_self:
        keep = src != dst
        src, dst = src[keep], dst[keep]
    key = torch.unique(src.to(torch.int64) * (V + 1) + dst.to(torch.int64))
    s = key // (V + 1)
    return s, key - s * (V + 1)


# ----------------------------------------------------------------------
# generators (return V, src, dst as int64 tensors, 1-based)
# ----------------------------------------------------------------------
def planted_random(V: int = 1024, m: int = 8192, n_cycles: int = 16, lmin: int = 4, lmax: int = 32,
                   seed: int = 1, device="cpu") -> Tuple[int, torch.Tensor, torch.Tensor]:
    g = _gen(seed, device)
    src = torch.randint(1, V + 1, (m,), generator=g, device=device)
    dst = torch.randint(1, V + 1, (m,), generator=g, device=device)
    cs, cd = [src], [dst]
    for _ in range(n_cycles):
        L = int(torch.randint(lmin, lmax + 1, (1,), generator=g, device=device).item())
        verts = torch.randperm(V, generator=g, device=device)[:L] + 1
        cs.append(verts)
        cd.append(torch.roll(verts, -1))
    return V, torch.cat(cs), torch.cat(cd)


def rmat(scale: int = 22, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 1, device="cpu",
         clean: bool = True, permute: bool = False) -> Tuple[int, torch.Tensor, torch.Tensor]:
    """R-MAT arcs.  With permute, vertex ids are relabelled by a seeded random
    permutation (as Graph500 does), so that ids no longer follow degree: the
    unpermuted generator gives the hubs the lowest ids."""
    V = 1 << scale
    m = edge_factor * V
    g = _gen(seed, device)
    u = torch.zeros(m, dtype=torch.int64, device=device)
    v = torch.zeros(m, dtype=torch.int64, device=device)
    ab, abc = a + b, a + b + c
    for bit in range(scale - 1, -1, -1):
        r = torch.rand(m, generator=g, device=device)
        ub = (r >= ab).to(torch.int64)                       # quadrants c, d
        vb = (((r >= a) & (r < ab)) | (r >= abc)).to(torch.int64)  # quadrants b, d
        u |= ub << bit
        v |= vb << bit
    if permute:
        perm = torch.randperm(V, generator=_gen(seed + 7919, device), device=device)
        u, v = perm[u], perm[v]
    u += 1
    v += 1
    if clean:
        u, v = dedup(V, u, v, drop_self=True)
    return V, u, v


def grid(n: int = 4096, p_bidir: float = 0.7, long_frac: float = 0.001, seed: int = 1,
         device="cpu") -> Tuple[int, torch.Tensor, torch.Tensor]:
    V = n * n
    g = _gen(seed, device)
    idx = torch.arange(V, dtype=torch.int64, device=device).view(n, n)
    a_h, b_h = idx[:, :-1].reshape(-1), idx[:, 1:].reshape(-1)   # right neighbours
    a_v, b_v = idx[:-1, :].reshape(-1), idx[1:, :].reshape(-1)   # down neighbours
    a = torch.cat([a_h, a_v]) + 1
    b = torch.cat([b_h, b_v]) + 1
    r = torch.rand(a.shape[0], generator=g, device=device)
    bi = r < p_bidir
    flip = torch.rand(a.shape[0], generator=g, device=device) < 0.5
    one_src = torch.where(flip, b, a)
    one_dst = torch.where(flip, a, b)
    src = torch.cat([a[bi], b[bi], one_src[~bi]])
    dst = torch.cat([b[bi], a[bi], one_dst[~bi]])
    n_long = int(round(long_frac * src.shape[0]))
    ls = torch.randint(1, V + 1, (n_long,), generator=g, device=device)
    ld = torch.randint(1, V + 1, (n_long,), generator=g, device=device)
    keep = ls != ld
    return V, torch.cat([src, ls[keep]]), torch.cat([dst, ld[keep]])


def _planted_chain(V: int, deg: float, rng: np.random.Generator) -> Tuple[np.ndarray, np.ndarray]:
    """k strongly connected blocks (cycle + chords) linked acyclically."""
    k = int(rng.integers(2, max(3, V // 8)))
    cuts = np.sort(rng.choice(np.arange(1, V), size=min(k - 1, V - 1), replace=False))
    bounds = np.concatenate([[0], cuts, [V]]).astype(np.int64)
    nb = len(bounds) - 1
    perm = rng.permutation(V).astype(np.int64) + 1
    start = np.repeat(bounds[:-1], np.diff(bounds))          # block start of every position
    end = np.repeat(bounds[1:], np.diff(bounds))
    pos = np.arange(V, dtype=np.int64)
    nxt = np.where(pos + 1 < end, pos + 1, start)             # cycle inside each block
    multi = (end - start) > 1
    srcs, dsts = [perm[pos[multi]]], [perm[nxt[multi]]]
    # chords inside blocks: a random position, then a random position of the same block
    n_ch = int(V * max(deg - 2.0, 0.0) * 0.5)
    if n_ch:
        p1 = rng.integers(0, V, n_ch)
        p2 = start[p1] + (rng.random(n_ch) * (end[p1] - start[p1])).astype(np.int64)
        srcs.append(perm[p1])
        dsts.append(perm[p2])
    # acyclic links from a block to a later block
    n_links = int(V * min(deg, 4.0) * 0.5)
    bi = rng.integers(0, nb, n_links)
    bj = rng.integers(0, nb, n_links)
    lo, hi = np.minimum(bi, bj), np.maximum(bi, bj)
    ok = lo < hi
    lo, hi = lo[ok], hi[ok]
    su = perm[bounds[lo] + (rng.random(len(lo)) * (bounds[lo + 1] - bounds[lo])).astype(np.int64)]
    sv = perm[bounds[hi] + (rng.random(len(hi)) * (bounds[hi + 1] - bounds[hi])).astype(np.int64)]
    srcs.append(su)
    dsts.append(sv)
    return np.concatenate(srcs), np.concatenate(dsts)


def batch_mix_sizes(n_graphs: int = 4096, vmin: int = 64, vmax: int = 65536, dmin: float = 4.0,
                    dmax: float = 16.0, seed: int = 1) -> List[Tuple[int, float]]:
    """(V, mean out-degree) of every graph of the mix, without building any."""
    out = []
    for i in range(n_graphs):
        rng = np.random.default_rng([seed, i])
        V = int(round(math.exp(rng.uniform(math.log(vmin), math.log(vmax)))))
        out.append((V, float(rng.uniform(dmin, dmax))))
    return out


def batch_mix_graph(i: int, vmin: int = 64, vmax: int = 65536, dmin: float = 4.0, dmax: float = 16.0,
                    seed: int = 1) -> Tuple[int, np.ndarray, np.ndarray]:
    """Graph i of the mix as (V, src, dst) numpy arcs.  Every graph has its
    own generator (seeded by (seed, i)), so any subset can be built alone."""
    rng = np.random.default_rng([seed, i])
    V = int(round(math.exp(rng.uniform(math.log(vmin), math.log(vmax)))))
    deg = float(rng.uniform(dmin, dmax))
    if i % 2 == 0:
        m = int(round(V * deg))
        s = rng.integers(1, V + 1, m)
        d = rng.integers(1, V + 1, m)
    else:
        s, d = _planted_chain(V, deg, rng)
    return V, s, d


def batch_mix_bytes(V: int, deg: float) -> int:
    """Estimated forward + reverse CSR bytes of a mix graph (for sharding)."""
    return 4 * (2 * (V + 2) + 2 * int(round(V * deg)))


def batch_mix(n_graphs: int = 4096, vmin: int = 64, vmax: int = 65536, dmin: float = 4.0,
              dmax: float = 16.0, seed: int = 1) -> List[Tuple[int, np.ndarray, np.ndarray]]:
    """List of (V, src, dst) numpy arcs for the batched configuration."""
    return [batch_mix_graph(i, vmin, vmax, dmin, dmax, seed) for i in range(n_graphs)]


def random_graph(V: int, m: int, seed: int = 0) -> Tuple[int, np.ndarray, np.ndarray]:
    rng = np.random.default_rng(seed)
    return V, rng.integers(1, V + 1, m), rng.integers(1, V + 1, m)
