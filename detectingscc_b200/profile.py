"""Short, self-contained workloads for capturing one kernel family under a
profiler: graphs are generated on the host (no device kernels run before the
profiled ones apart from copies), inputs of the default sizes are larger than
the 126 MB L2, and each run holds a few GB of device memory at most.

    python -m detectingscc_b200.profile derive [--scale 22] [--reps 2]
        scc_derive_reverse on the R-MAT graph of that scale
        (k_tr_tile_owner, k_tr_expand, k_rs_hist, k_tile_*, k_scan_sums,
        k_rs_scatter, k_tr_offsets)
    python -m detectingscc_b200.profile ingest [--scale 20] [--reps 2]
        scc_load_graph_device on the R-MAT graph written as GTgraph text
        (k_parse_count, k_parse_write and the sorts above)
    python -m detectingscc_b200.profile scc --config cfg1|cfg2|cfg3 [--reps 2]
        one decomposition per rep (k_scc_block or k_scc_grid, k_canon_write)
    python -m detectingscc_b200.profile batch [--graphs 256] [--reps 2]
        the batched form on the largest graphs of the 4,096-graph mix
        (k_scc_batch), default schedule

Every run checks its result against the host-built CSR or the oracle-free
invariants it can (derive: bit-exact reverse CSR; ingest: bit-exact CSRs;
scc/batch: SCC count equal on every rep) and prints one line per rep.  It is
a profiling aid, not a benchmark: bench.py measures.
"""
from __future__ import annotations

import argparse
import os
import tempfile
import time

import numpy as np


def _graph(kind: str, scale: int):
    import detectingscc_b200 as scc
    from detectingscc_b200 import graphs
    if kind == "cfg1":
        V, s, d = graphs.planted_random(seed=1)
    elif kind == "cfg3":
        V, s, d = graphs.grid(scale or 4096, seed=1)
    else:
        V, s, d = graphs.rmat(scale or 22, seed=1)
    return scc.graph_from_arcs(V, s.numpy(), d.numpy())


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def run_derive(args):
    import torch

    import detectingscc_b200 as scc
    g = _graph("rmat", args.scale)
    Fr, Fc = _dev(g.Fr), _dev(g.Fc)
    Br = torch.empty(g.V + 2, dtype=torch.int32, device="cuda")
    Bc = torch.empty(max(g.E, 1), dtype=torch.int32, device="cuda")
    eng = scc.Engine(0)
    for r in range(args.reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.derive_reverse(g.V, g.E, Fr, Fc, Br, Bc)
        torch.cuda.synchronize()
        print(f"derive rep {r}: V={g.V} E={g.E} {1e3 * (time.perf_counter() - t0):.3f} ms", flush=True)
    assert np.array_equal(Br.cpu().numpy().view(np.uint32), g.Br)
    assert np.array_equal(Bc.cpu().numpy().view(np.uint32)[:g.E], g.Bc)
    eng.close()


def run_ingest(args):
    import torch

    import detectingscc_b200 as scc
    g = _graph("rmat", args.scale or 20)
    path = os.path.join(tempfile.gettempdir(), f"sccb_profile_{os.getpid()}.gr")
    scc.save_gtgraph(path, g)
    eng = scc.Engine(0)
    try:
        for r in range(args.reps):
            t0 = time.perf_counter()
            V, E, Fr, Fc, Br, Bc = eng.load_graph_device(path)
            torch.cuda.synchronize()
            print(f"ingest rep {r}: V={V} E={E} {1e3 * (time.perf_counter() - t0):.1f} ms", flush=True)
        out = torch.empty(max(V, 1), dtype=torch.int32, device="cuda")
        res = eng.run_device(V, E, Fr, Fc, Br, Bc, labels_out=out, algo="h")
        ref = eng.run(g, algo="h")
        assert res.num_sccs == ref.num_sccs
    finally:
        os.remove(path)
        eng.close()


def run_scc(args):
    import torch

    import detectingscc_b200 as scc
    algo = {"cfg1": ("g", True, False, 1), "cfg2": ("h", True, True, 1), "cfg3": ("y", True, True, 8)}[args.config]
    g = _graph(args.config, args.scale)
    tens = [_dev(a) for a in (g.Fr, g.Fc, g.Br, g.Bc)]
    out = torch.empty(g.V, dtype=torch.int32, device="cuda")
    eng = scc.Engine(0)
    n0 = None
    for r in range(args.reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = eng.run_device(g.V, g.E, *tens, labels_out=out, algo=algo[0], t1=algo[1], t2=algo[2], warp=algo[3])
        torch.cuda.synchronize()
        n0 = res.num_sccs if n0 is None else n0
        assert res.num_sccs == n0
        print(f"scc {args.config} rep {r}: V={g.V} E={g.E} sccs={res.num_sccs} "
              f"{1e3 * (time.perf_counter() - t0):.3f} ms", flush=True)
    eng.close()


def run_batch(args):
    import detectingscc_b200 as scc
    from detectingscc_b200 import graphs
    sizes = graphs.batch_mix_sizes(4096, seed=1)
    idx = sorted(range(4096), key=lambda i: -sizes[i][0])[:args.graphs]
    gs = [scc.graph_from_arcs(*graphs.batch_mix_graph(i, seed=1)) for i in idx]
    eng = scc.Engine(0)
    b = scc.Batch(eng, gs)
    try:
        n0 = None
        for r in range(args.reps):
            t0 = time.perf_counter()
            _, res, _ = b.run(algo="g", t1=True, t2=True, labels=False)
            n = sum(x[0] for x in res)
            n0 = n if n0 is None else n0
            assert n == n0 and all(x[2] == 0 for x in res)
            print(f"batch rep {r}: {len(gs)} graphs, {n} SCCs, {1e3 * (time.perf_counter() - t0):.2f} ms", flush=True)
    finally:
        b.close()
        eng.close()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("what", choices=["derive", "ingest", "scc", "batch"])
    ap.add_argument("--scale", type=int, default=None)
    ap.add_argument("--config", default="cfg2", choices=["cfg1", "cfg2", "cfg3"])
    ap.add_argument("--graphs", type=int, default=256)
    ap.add_argument("--reps", type=int, default=2)
    args = ap.parse_args()
    {"derive": run_derive, "ingest": run_ingest, "scc": run_scc, "batch": run_batch}[args.what](args)


if __name__ == "__main__":
    main()
