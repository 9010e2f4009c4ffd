"""Bit-exact parity at the five benchmark configurations' full sizes.

Each test builds the configuration's graph exactly as bench.py does (same
generator, seed and device), runs it through the public API and compares
every vertex's canonical label (smallest vertex id of its SCC) with the
oracle's iterative Tarjan: integer labels, tolerance 0.  Counters are pinned
too: for the Slota drivers the reference counts trim-1 SCCs (one trim pass
over the whole graph, scc_Coloring.cu:507-508, so exactly the vertices with
no in- or no out-arc) and pivots (every other SCC, scc_Coloring.cu:640-652);
for vHong on cfg1 the restated reference schedule gives all three counters.

cfg1  vHong -p 1 -q 0, 1,024 vertices + 8,192 arcs + 16 planted cycles, seed 1
cfg2  vSlota -p 1 -q 1, R-MAT scale 22, edge factor 16, seed 1 (and the same
      graph with its vertex ids randomly permuted)
cfg3  wSlota -w 8, 4096 x 4096 grid, seed 1
cfg4  a slice of the 4,096-graph mix holding its largest graphs (planted
      chains and Erdos-Renyi graphs up to ~65K vertices), autotuned schedule
      and a forced cluster schedule, labels read back
cfg5  the serving pool's R-MAT scale-20 graph served in a mix of small ones
"""
import numpy as np
import pytest

import detectingscc_b200 as scc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = scc.Engine(0)
    yield e
    e.close()


def _device_graph(gen):
    import torch

    from detectingscc_b200 import graphs
    V, s, d = gen(torch.device("cuda", 0))
    Fr, Fc, Br, Bc = graphs.csr_from_arcs_torch(V, s, d)
    del s, d
    return V, Fr, Fc, Br, Bc


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def _slota_counts(Fr, Br, V):
    indeg = np.diff(Br.astype(np.int64))[1:V + 1]
    outdeg = np.diff(Fr.astype(np.int64))[1:V + 1]
    return int(np.count_nonzero((indeg == 0) | (outdeg == 0)))


def _run_and_check(engine, oracle_lib, V, Fr, Fc, Br, Bc, algo, t1, t2, warp):
    import torch
    E = int(Fc.shape[0])
    out = torch.empty(V, dtype=torch.int32, device=Fr.device)
    res = engine.run_device(V, E, Fr, Fc, Br, Bc, labels_out=out, algo=algo, t1=t1, t2=t2, warp=warp)
    hFr, hFc = _host(Fr), _host(Fc)
    lab, n = oracle_lib.tarjan(V, hFr, hFc)
    got = _host(out)
    bad = np.flatnonzero(got != lab[1:])
    assert bad.size == 0, f"{bad.size} labels differ, first at vertex {bad[0] + 1}: {got[bad[0]]} vs {lab[bad[0] + 1]}"
    assert res.num_sccs == n
    return res, hFr, _host(Br), n


def test_cfg1_vhong_planted_random(engine, oracle_lib):
    from detectingscc_b200 import graphs
    V, Fr, Fc, Br, Bc = _device_graph(lambda dev: graphs.planted_random(seed=1, device=dev))
    res, hFr, hBr, n = _run_and_check(engine, oracle_lib, V, Fr, Fc, Br, Bc, "g", True, False, 1)
    _, counts = oracle_lib.hong(V, hFr, _host(Fc), hBr, _host(Bc), True, False)
    assert [res.num_trim1, res.num_trim2, res.num_pivot] == counts


@pytest.mark.parametrize("permute", [False, True])
def test_cfg2_vslota_rmat22(engine, oracle_lib, permute):
    from detectingscc_b200 import graphs
    V, Fr, Fc, Br, Bc = _device_graph(lambda dev: graphs.rmat(22, seed=1, device=dev, permute=permute))
    assert V == 1 << 22
    res, hFr, hBr, n = _run_and_check(engine, oracle_lib, V, Fr, Fc, Br, Bc, "h", True, True, 1)
    t1 = _slota_counts(hFr, hBr, V)
    assert [res.num_trim1, res.num_trim2, res.num_pivot] == [t1, 0, n - t1]


def test_cfg2_reverse_csr_built_on_the_device(engine):
    """The device-built reverse CSR of the R-MAT scale-22 graph equals the
    reference loader's layout (in-lists in ascending source order)."""
    import torch

    from detectingscc_b200 import graphs
    V, Fr, Fc, Br, Bc = _device_graph(lambda dev: graphs.rmat(22, seed=1, device=dev))
    E = int(Fc.shape[0])
    dBr = torch.full_like(Br, -1)
    dBc = torch.full_like(Bc, -1)
    engine.derive_reverse(V, E, Fr, Fc, dBr, dBc)
    torch.cuda.synchronize()
    assert torch.equal(dBr, Br) and torch.equal(dBc, Bc)


def test_cfg3_wslota_grid4096(engine, oracle_lib):
    from detectingscc_b200 import graphs
    V, Fr, Fc, Br, Bc = _device_graph(lambda dev: graphs.grid(4096, seed=1, device=dev))
    assert V == 4096 * 4096
    res, hFr, hBr, n = _run_and_check(engine, oracle_lib, V, Fr, Fc, Br, Bc, "y", True, True, 8)
    t1 = _slota_counts(hFr, hBr, V)
    assert [res.num_trim1, res.num_trim2, res.num_pivot] == [t1, 0, n - t1]


def _cfg4_slice(n_each=32):
    """Indices of the cfg4 mix (4,096 graphs, seed 1): its n_each largest
    planted chains, its n_each largest Erdos-Renyi graphs and n_each more
    spread over the size range."""
    from detectingscc_b200 import graphs
    sizes = graphs.batch_mix_sizes(4096, seed=1)
    chains = sorted(range(1, 4096, 2), key=lambda i: -sizes[i][0])[:n_each]
    er = sorted(range(0, 4096, 2), key=lambda i: -sizes[i][0])[:n_each]
    rest = [i for i in range(0, 4096, 4096 // n_each) if i not in chains and i not in er]
    return sorted(set(chains + er + rest)), sizes


def test_cfg4_slice_batched(engine, oracle_lib):
    from detectingscc_b200 import graphs
    idx, sizes = _cfg4_slice()
    assert max(sizes[i][0] for i in idx) > 60000
    gs = [scc.graph_from_arcs(*graphs.batch_mix_graph(i, seed=1)) for i in idx]
    ref = [oracle_lib.tarjan(g.V, g.Fr, g.Fc) for g in gs]
    b = scc.Batch(engine, gs)
    try:
        b.autotune(algo="g")                      # as the benchmark does
        schedules = [b.cluster()[:2], (4, 16384), (8, 32768)]
        for cl, big in schedules:
            b.set_cluster(cl, big)
            labels, res, _ = b.run(algo="g", t1=True, t2=True)
            for k, g in enumerate(gs):
                lab, n = ref[k]
                assert res[k][2] == 0 and res[k][0] == n, (cl, big, idx[k])
                assert np.array_equal(b.labels_of(labels, k), lab[1:]), (cl, big, idx[k])
    finally:
        b.close()


def test_cfg5_rmat20_served_in_a_mix(oracle_lib):
    import time

    import torch

    from detectingscc_b200 import graphs
    V, s, d = graphs.rmat(20, seed=100, device=torch.device("cuda", 0))
    large = graphs.to_graph(V, s, d)
    small = [scc.graph_from_arcs(*graphs.batch_mix_graph(i, seed=11)) for i in range(64)]
    pool = small + [large]
    srv = scc.Server(0, algo="g", t1=True, t2=True, budget_bytes=120 * 10**9)
    try:
        tickets = {}
        for k in range(len(pool)):
            tickets[srv.submit(pool[k])] = k
            if k == 8:
                tickets[srv.submit(large)] = len(pool) - 1   # the large graph twice, once early
        got = {}
        t0 = time.time()
        while len(got) < len(tickets) and time.time() - t0 < 300:
            for r in srv.poll(256, wait_ms=200):
                got[r["ticket"]] = r
        assert len(got) == len(tickets)
        for t, k in tickets.items():
            r = got[t]
            assert r["status"] == 0, r
            lab, n = oracle_lib.tarjan(pool[k].V, pool[k].Fr, pool[k].Fc)
            assert np.array_equal(r["labels"], lab[1:]), k
    finally:
        srv.close()
