"""Batched form: many graphs in one launch, each graph's labels bit-exact
against Tarjan and equal to the per-graph plain path; a malformed graph
fails alone."""
import numpy as np
import pytest

import detectingscc_b200 as scc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = scc.Engine(0)
    yield e
    e.close()


def _mix(n, seed, vmax=3000):
    from detectingscc_b200 import graphs
    out = []
    for V, s, d in graphs.batch_mix(n, vmin=16, vmax=vmax, seed=seed):
        out.append(scc.graph_from_arcs(V, s, d))
    return out


@pytest.mark.parametrize("algo,w", [("h", 1), ("g", 1), ("y", 8), ("x", 4)])
def test_batch_matches_tarjan_and_plain(engine, oracle_lib, algo, w):
    gs = _mix(96, seed=3)
    gs.append(scc.graph_from_arcs(1, [], []))          # single isolated vertex
    b = scc.Batch(engine, gs)
    try:
        labels, res, st = b.run(algo=algo, warp=w)
        seq_labels, seq_res, _ = b.run(algo=algo, warp=w, sequential=True)
        assert np.array_equal(labels, seq_labels)
        for i, g in enumerate(gs):
            ref, n = oracle_lib.tarjan(g.V, g.Fr, g.Fc)
            assert np.array_equal(b.labels_of(labels, i), ref[1:]), i
            assert res[i][0] == n and res[i][2] == 0
            assert seq_res[i][0] == n
        # replays of the captured launch give the same answer
        again, _, _ = b.run(algo=algo, warp=w)
        assert np.array_equal(again, labels)
    finally:
        b.close()


def test_batch_schedules_and_autotune(engine, oracle_lib):
    gs = _mix(40, seed=5)
    b = scc.Batch(engine, gs)
    try:
        ref = [oracle_lib.tarjan(g.V, g.Fr, g.Fc)[0][1:] for g in gs]
        for threads, q in [(128, 64), (256, 256), (512, 128), (1024, 512)]:
            b.set_schedule(threads, q)
            labels, res, _ = b.run(algo="h")
            for i in range(len(gs)):
                assert np.array_equal(b.labels_of(labels, i), ref[i])
        t, q, ms = b.autotune(algo="h")
        assert (t, q) == b.schedule() and ms > 0
    finally:
        b.close()


def test_bad_graph_fails_alone(engine, oracle_lib):
    gs = _mix(8, seed=7)
    bad = scc.graph_from_arcs(5, [1, 2, 3], [2, 3, 1])
    bad.Fc[0] = 99                                      # id outside [1, V]
    gs.insert(3, bad)
    b = scc.Batch(engine, gs)
    try:
        labels, res, _ = b.run(algo="g", check=False)
        assert res[3][2] == 23                          # SCC_ERR_BAD_GRAPH
        for i, g in enumerate(gs):
            if i == 3:
                continue
            ref, n = oracle_lib.tarjan(g.V, g.Fr, g.Fc)
            assert res[i][2] == 0 and np.array_equal(b.labels_of(labels, i), ref[1:])
    finally:
        b.close()


@pytest.mark.parametrize("algo,w", [("g", 1), ("h", 1), ("y", 8)])
def test_cluster_graphs_match_tarjan(engine, oracle_lib, algo, w):
    """Graphs run on whole thread-block clusters (every cluster size) give
    the same labels as one CTA per graph and as Tarjan: first with the
    bounded software cluster barrier (check mode), then the hardware one."""
    gs = _mix(40, seed=7, vmax=6000)
    gs.append(scc.graph_from_arcs(1, [], []))
    ref = [oracle_lib.tarjan(g.V, g.Fr, g.Fc)[0][1:] for g in gs]
    for check in (1, 0):
        engine.set_tuning("cluster_check", check)
        b = scc.Batch(engine, gs)
        try:
            base, _, _ = b.run(algo=algo, warp=w)
            for cl, big in [(2, 0), (4, 1000), (8, 2000), (16, 0)]:
                b.set_cluster(cl, big)
                c, bv, nb = b.cluster()
                assert (c, bv) == (cl, big) and nb == sum(g.V >= big for g in gs)
                labels, res, _ = b.run(algo=algo, warp=w)
                assert all(r[2] == 0 for r in res), (check, cl, res)
                assert np.array_equal(labels, base)
                for i in range(len(gs)):
                    assert np.array_equal(b.labels_of(labels, i), ref[i]), (check, cl, big, i)
            b.set_cluster(1, 0)
            again, _, _ = b.run(algo=algo, warp=w)
            assert np.array_equal(again, base)
        finally:
            b.close()
            engine.set_tuning("cluster_check", 0)
