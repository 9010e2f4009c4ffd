"""CUDA engine vs the oracle, through the C ABI, on a B200.

Integer work: labels must be bit-exact (tolerance 0) against Tarjan /
the golden fixtures, and the counters (trim-1, trim-2, pivot SCCs) must
equal the restated reference schedule's counters exactly.
"""
import numpy as np
import pytest

import detectingscc_b200 as scc
from conftest import SAMPLES
from golden_graphs import csr, edge_cases
from oracle.gtgraph_ref import build_csr

pytestmark = pytest.mark.gpu

ALGO_CASES = [("g", 1), ("h", 1), ("x", 1), ("x", 8), ("x", 32), ("y", 1), ("y", 4), ("y", 8), ("y", 32)]


@pytest.fixture(scope="module")
def engine():
    e = scc.Engine(0)
    yield e
    e.close()


def _graph(V, Fr, Fc, Br, Bc):
    return scc.Graph(V, int(Fr[-1]), Fr, Fc, Br, Bc)


def _expect(oracle_lib, g, algo, t1, t2):
    fn = oracle_lib.hong if algo in "gx" else oracle_lib.slota
    lab, counts = fn(g.V, g.Fr, g.Fc, g.Br, g.Bc, t1, t2)
    return lab[1:], counts


def _check(engine, oracle_lib, g, algo, w, t1, t2, force=None):
    res = engine.run(g, algo=algo, t1=t1, t2=t2, warp=w, force=force)
    lab, counts = _expect(oracle_lib, g, algo, t1, t2)
    assert np.array_equal(res.labels, lab), (algo, w, t1, t2, force)
    assert [res.num_trim1, res.num_trim2, res.num_pivot] == counts, (algo, w, t1, t2, force)
    assert res.num_sccs == sum(counts)
    return res


@pytest.mark.parametrize("name", SAMPLES)
@pytest.mark.parametrize("algo,w", ALGO_CASES)
@pytest.mark.parametrize("t1,t2", [(1, 1), (1, 0), (0, 1), (0, 0)])
def test_golden_fixtures(engine, oracle_lib, golden, name, algo, w, t1, t2):
    z = golden[name]
    V = int(z["V"])
    g = _graph(V, *build_csr(V, z["src"].astype(np.int64), z["dst"].astype(np.int64)))
    res = _check(engine, oracle_lib, g, algo, w, t1, t2)
    assert np.array_equal(res.labels, z["labels"])
    assert res.num_sccs == int(z["nscc"])


@pytest.mark.parametrize("force", ["grid", "block"])
@pytest.mark.parametrize("case", edge_cases(), ids=lambda c: c[0])
def test_edge_cases_both_launch_paths(engine, oracle_lib, case, force):
    name, V, s, d = case
    arcs = np.stack([np.asarray(s, np.int64), np.asarray(d, np.int64)], 1) if len(s) else np.zeros((0, 2), np.int64)
    g = _graph(*csr(V, arcs))
    for algo, w in [("g", 1), ("h", 1), ("x", 4), ("y", 8)]:
        for t1, t2 in [(1, 1), (0, 0), (1, 0)]:
            _check(engine, oracle_lib, g, algo, w, t1, t2, force=force)


@pytest.mark.parametrize("gen", ["rmat14", "grid128", "planted"])
def test_generated_graphs_grid_path(engine, oracle_lib, gen):
    from detectingscc_b200 import graphs
    V, s, d = {"rmat14": lambda: graphs.rmat(14, seed=3), "grid128": lambda: graphs.grid(128, seed=4),
               "planted": lambda: graphs.planted_random(seed=9)}[gen]()
    g = graphs.to_graph(V, s, d)
    for algo, w in [("g", 1), ("h", 1), ("x", 8), ("y", 8)]:
        _check(engine, oracle_lib, g, algo, w, 1, 1, force="grid")
        _check(engine, oracle_lib, g, algo, w, 1, 0, force="grid")


def test_tail_switch_to_one_cta(engine, oracle_lib):
    from detectingscc_b200 import graphs
    try:
        engine.set_tuning("tail_vertices", 1 << 30)
        for gen in (lambda: graphs.rmat(13, seed=11), lambda: graphs.grid(64, seed=3)):
            V, s, d = gen()
            g = graphs.to_graph(V, s, d)
            for algo in ("g", "h"):
                for t1, t2 in ((1, 1), (0, 0)):
                    res = _check(engine, oracle_lib, g, algo, 1, t1, t2, force="grid")
                    # CTA 0 takes over at the first main-loop iteration / peel
                    assert res.stats["outer_iters"] == 0 or res.stats["tail_pass"] > 0
    finally:
        engine.set_tuning("tail_vertices", 1024)


def test_repeatable(engine, oracle_lib):
    from detectingscc_b200 import graphs
    V, s, d = graphs.rmat(15, seed=1)
    g = graphs.to_graph(V, s, d)
    a = engine.run(g, algo="h", force="grid")
    b = engine.run(g, algo="h", force="grid")
    assert np.array_equal(a.labels, b.labels) and a.num_sccs == b.num_sccs


def test_bad_column_id_is_reported(engine):
    V, Fr, Fc, Br, Bc = csr(4, [[1, 2], [2, 1], [3, 4]])
    Fc = Fc.copy()
    Fc[0] = 9  # outside [1, V]
    g = _graph(V, Fr, Fc, Br, Bc)
    with pytest.raises(scc.SCCError) as e:
        engine.run(g, algo="h")
    assert e.value.code == 23
    # the context stays usable
    V, Fr, Fc, Br, Bc = csr(4, [[1, 2], [2, 1], [3, 4]])
    assert engine.run(_graph(V, Fr, Fc, Br, Bc), algo="g").num_sccs == 3


def test_bad_offsets_are_reported(engine):
    V, Fr, Fc, Br, Bc = csr(4, [[1, 2], [2, 1], [3, 4]])
    Fr = Fr.copy()
    Fr[2], Fr[3] = Fr[3], Fr[2] + 5
    g = scc.Graph(V, 3, Fr, Fc, Br, Bc)
    with pytest.raises(scc.SCCError) as e:
        engine.run(g, algo="g")
    assert e.value.code == 23


def test_invalid_arguments(engine):
    V, Fr, Fc, Br, Bc = csr(3, [[1, 2]])
    g = _graph(V, Fr, Fc, Br, Bc)
    with pytest.raises(scc.SCCError) as e:
        engine.run(g, algo="y", warp=3)
    assert e.value.code == 1
    with pytest.raises(ValueError):
        engine.run(g, algo="q")


def test_instrumented_counters(engine, oracle_lib):
    from detectingscc_b200 import graphs
    V, s, d = graphs.rmat(12, seed=2)
    g = graphs.to_graph(V, s, d)
    res = engine.run(g, algo="h", instrument=True, force="grid")
    assert res.stats["edges_scanned"] > 0 and res.stats["vertex_visits"] >= g.V
    lab, _ = _expect(oracle_lib, g, "h", 1, 1)
    assert np.array_equal(res.labels, lab)


def test_device_resident_path(engine, oracle_lib):
    import torch
    from detectingscc_b200 import graphs
    V, s, d = graphs.rmat(14, seed=6, device="cuda")
    Fr, Fc, Br, Bc = graphs.csr_from_arcs_torch(V, s, d)
    out = torch.empty(V, dtype=torch.int32, device="cuda")
    res = engine.run_device(V, Fc.shape[0], Fr, Fc, Br, Bc, labels_out=out, algo="h")
    g = scc.Graph(V, int(Fc.shape[0]), Fr.cpu().numpy(), Fc.cpu().numpy(), Br.cpu().numpy(), Bc.cpu().numpy())
    lab, counts = _expect(oracle_lib, g, "h", 1, 1)
    assert np.array_equal(out.cpu().numpy().astype(np.uint32), lab)
    assert res.num_sccs == sum(counts)


@pytest.mark.parametrize("sched", [1, 2])
@pytest.mark.parametrize("algo,w", [("x", 1), ("x", 8), ("y", 2), ("y", 8), ("y", 32)])
def test_warp_schedules(oracle_lib, golden, sched, algo, w):
    """wHong / wSlota with the virtual-warp schedule forced (1) and the warp
    walk forced (2): the same labels and counters as the restated reference,
    on both launch paths (the default picks one by mean degree)."""
    from detectingscc_b200 import graphs
    e = scc.Engine(0)
    e.set_tuning("warp_schedule", sched)
    try:
        gs = []
        for name in SAMPLES:
            z = golden[name]
            V = int(z["V"])
            gs.append(_graph(V, *build_csr(V, z["src"].astype(np.int64), z["dst"].astype(np.int64))))
        for gen in (lambda: graphs.grid(64, seed=2), lambda: graphs.rmat(12, seed=6)):
            V, s, d = gen()
            gs.append(scc.graph_from_arcs(V, s.numpy(), d.numpy()))
        for g in gs:
            for force in ("grid", "block"):
                _check(e, oracle_lib, g, algo, w, 1, 1, force)
    finally:
        e.close()


@pytest.mark.parametrize("algo,w", [("h", 1), ("y", 8), ("g", 1)])
def test_direction_rule(oracle_lib, algo, w):
    """The frontier-edge tally behind the bottom-up rule is skipped on passes
    whose claims cannot reach the threshold (claims x maximum degree): labels
    and counters match the restated reference with bottom-up steps allowed
    and switched off, R-MAT still takes bottom-up steps on the whole-GPU
    kernel, and the low-degree grid takes none."""
    from detectingscc_b200 import graphs
    e = scc.Engine(0)
    e.set_tuning("trace", 4096)
    try:
        for gen, hubs in ((lambda: graphs.rmat(16, seed=4), True), (lambda: graphs.grid(192, seed=5), False)):
            V, s, d = gen()
            g = scc.graph_from_arcs(V, s.numpy(), d.numpy())
            for bu in (2, 0):
                e.set_tuning("bu_k", bu)
                _check(e, oracle_lib, g, algo, w, 1, 1, "grid")
                pulled = any(p == "bfs_pull" for p, _, _ in e.trace())
                assert pulled == (hubs and bu > 0), (algo, w, bu, hubs)
    finally:
        e.close()
