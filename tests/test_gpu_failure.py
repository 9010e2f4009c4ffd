"""Failure detection on the GPU without faulting it.

Every device-side wait and convergence loop of the engine is bounded and
ends in an error status the host reads (the reference's host loops have no
bound at all: scc_WCC.cu:851-930).  These tests make each bound run out on
purpose and check the status and that the context stays usable:

* a pass cap of 2 on a long chain: SCC_ERR_NOT_CONVERGED (21);
* one CTA withholding its grid-barrier arrival (an arrival that never
  comes) with a 50 ms wait bound: SCC_ERR_TIMEOUT (22) from the whole-GPU
  launch;
* the same in a batched launch whose big graphs run on thread-block
  clusters with the bounded software cluster barrier (check mode): those
  graphs fail with SCC_ERR_TIMEOUT, the graphs on single CTAs do not.

Nothing here traps, asserts on the device or waits without a bound.
"""
import numpy as np
import pytest

import detectingscc_b200 as scc

pytestmark = pytest.mark.gpu

NOT_CONVERGED, TIMEOUT = 21, 22


@pytest.fixture(scope="module")
def engine():
    e = scc.Engine(0)
    yield e
    e.close()


def _chain(n):
    src = np.arange(1, n, dtype=np.int64)
    return scc.graph_from_arcs(n, src, src + 1)


def _restore(engine):
    engine.set_tuning("max_passes", 0)
    engine.set_tuning("test_withhold_arrival", 0)
    engine.set_tuning("timeout_ms", 4000)
    engine.set_tuning("cluster_check", 0)


@pytest.mark.parametrize("force", ["grid", "block"])
def test_pass_cap_ends_in_not_converged(engine, oracle_lib, force):
    g = _chain(5000)      # without trim-1 every BFS level is one pass: thousands of passes
    try:
        engine.set_tuning("max_passes", 2)
        with pytest.raises(scc.SCCError) as e:
            engine.run(g, algo="g", t1=False, t2=False, force=force)
        assert e.value.code == NOT_CONVERGED
    finally:
        _restore(engine)
    # the context stays usable and the same graph now completes
    res = engine.run(g, algo="g", t1=False, t2=False, force=force)
    lab, n = oracle_lib.tarjan(g.V, g.Fr, g.Fc)
    assert res.num_sccs == n and np.array_equal(res.labels, lab[1:])


@pytest.mark.parametrize("at_pass", [1, 2])
def test_withheld_grid_arrival_ends_in_timeout(engine, oracle_lib, at_pass):
    from detectingscc_b200 import graphs
    V, s, d = graphs.rmat(14, seed=5)
    g = graphs.to_graph(V, s, d)
    try:
        engine.set_tuning("timeout_ms", 50)
        engine.set_tuning("test_withhold_arrival", at_pass)
        with pytest.raises(scc.SCCError) as e:
            engine.run(g, algo="h", force="grid")
        assert e.value.code == TIMEOUT
    finally:
        _restore(engine)
    res = engine.run(g, algo="h", force="grid")
    lab, n = oracle_lib.tarjan(g.V, g.Fr, g.Fc)
    assert res.num_sccs == n and np.array_equal(res.labels, lab[1:])


def test_withheld_cluster_arrival_fails_only_cluster_graphs(engine, oracle_lib):
    from detectingscc_b200 import graphs
    gs = [scc.graph_from_arcs(V, s, d) for V, s, d in graphs.batch_mix(24, vmin=16, vmax=6000, seed=13)]
    ref = [oracle_lib.tarjan(g.V, g.Fr, g.Fc)[0][1:] for g in gs]
    big = 2000
    b = scc.Batch(engine, gs)
    try:
        engine.set_tuning("cluster_check", 1)
        engine.set_tuning("timeout_ms", 50)
        engine.set_tuning("test_withhold_arrival", 2)
        b.set_cluster(4, big)
        _, res, _ = b.run(algo="h", check=False)
        on_cluster = [g.V >= big for g in gs]
        assert any(on_cluster) and not all(on_cluster)
        for i, r in enumerate(res):
            assert r[2] == (TIMEOUT if on_cluster[i] else 0), (i, gs[i].V, r)
        # bounds back to normal: every graph completes and matches Tarjan
        engine.set_tuning("test_withhold_arrival", 0)
        engine.set_tuning("timeout_ms", 4000)
        labels, res, _ = b.run(algo="h")
        for i in range(len(gs)):
            assert res[i][2] == 0 and np.array_equal(b.labels_of(labels, i), ref[i]), i
    finally:
        b.close()
        _restore(engine)
