"""Sharding of independent graphs across ranks (batched and serving forms):
the byte-balanced plan, and the host-side gather that puts every rank's
per-graph results back in global order, run as 2 gloo ranks on the CPU
(the per-rank solver here is the oracle's Tarjan; on GPUs it is a Batch)."""
import os
import socket

import numpy as np
import pytest

from detectingscc_b200.shard import gather_in_order, shard_by_bytes


def test_plan_covers_every_graph_once_and_balances():
    rng = np.random.default_rng(0)
    sizes = [int(x) for x in rng.integers(1, 10**6, 1000)]
    for world in (1, 2, 3, 8):
        plan = shard_by_bytes(sizes, world)
        flat = sorted(i for p in plan for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in plan]
        # greedy LPT: the spread is at most the largest item
        assert max(loads) - min(loads) <= max(sizes)
        assert plan == shard_by_bytes(sizes, world)          # deterministic


def test_plan_edge_cases():
    assert shard_by_bytes([], 3) == [[], [], []]
    assert shard_by_bytes([7], 2) == [[0], []]
    assert shard_by_bytes([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard_by_bytes([1], 0)


def test_gather_single_rank_and_mismatch():
    plan = shard_by_bytes([3, 1, 2], 1)
    assert gather_in_order(["a", "b", "c"], plan, 0) == ["a", "b", "c"]
    with pytest.raises(ValueError):
        gather_in_order(["a"], plan, 0)


def _solve(graphs):
    from oracle import oracle
    out = []
    for g in graphs:
        lab, n = oracle.tarjan(g.V, g.Fr, g.Fc)
        out.append((int(n), lab[1:].copy()))
    return out


def _build(i):
    import detectingscc_b200 as scc
    from detectingscc_b200 import graphs
    V, s, d = graphs.batch_mix_graph(i, vmin=16, vmax=3000, seed=4)
    return scc.graph_from_arcs(V, s, d)


def _sizes(n):
    from detectingscc_b200 import graphs
    return [graphs.batch_mix_bytes(V, deg) for V, deg in graphs.batch_mix_sizes(n, vmin=16, vmax=3000, seed=4)]


def _rank_main(rank, world, port, n, outdir):
    import torch.distributed as dist

    from detectingscc_b200.shard import run_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        full = run_sharded(_sizes(n), _build, _solve, rank, world)           # every rank gets all
        to0 = run_sharded(_sizes(n), _build, _solve, rank, world, dst=0)     # only rank 0
        assert (to0 is None) == (rank != 0)
        np.save(os.path.join(outdir, f"counts{rank}.npy"), np.array([c for c, _ in full]))
        np.save(os.path.join(outdir, f"labels{rank}.npy"), np.concatenate([lab for _, lab in full]))
        if rank == 0:
            np.save(os.path.join(outdir, "counts_dst.npy"), np.array([c for c, _ in to0]))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_reassemble_the_single_rank_answer(tmp_path):
    import torch.multiprocessing as mp
    from oracle import oracle
    oracle.build()
    n = 24
    mp.start_processes(_rank_main, args=(2, _free_port(), n, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    single = _solve([_build(i) for i in range(n)])
    want_counts = np.array([c for c, _ in single])
    want_labels = np.concatenate([lab for _, lab in single])
    for r in range(2):
        assert np.array_equal(np.load(tmp_path / f"counts{r}.npy"), want_counts)
        assert np.array_equal(np.load(tmp_path / f"labels{r}.npy"), want_labels)
    assert np.array_equal(np.load(tmp_path / "counts_dst.npy"), want_counts)


def _bench_rank_main(rank, world, port, n, outdir, device):
    """One rank of bench.py's cfg4 sharding: its plan, its shard built and
    solved (the batched engine on a GPU, else the oracle), the per-graph
    results gathered on rank 0 in global order."""
    import datetime

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        n_total, plan = bench.cfg4_plan(n, world)
        gs = bench._batch_graphs(n_total, seed=1, indices=plan[rank])
        if device:
            import detectingscc_b200 as scc
            eng = scc.Engine(0)
            b = scc.Batch(eng, gs)
            try:
                labels, res, _ = b.run(algo="g", t1=True, t2=True)
                counts = [int(r[0]) for r in res]
                labs = [b.labels_of(labels, k).copy() for k in range(len(gs))]
            finally:
                b.close()
                eng.close()
        else:
            sol = _solve(gs)
            counts, labs = [c for c, _ in sol], [lab for _, lab in sol]
        got_c = gather_in_order(counts, plan, rank, dst=0)
        got_l = gather_in_order(labs, plan, rank, dst=0)
        if rank == 0:
            np.save(os.path.join(outdir, "counts.npy"), np.array(got_c))
            np.save(os.path.join(outdir, "labels.npy"), np.concatenate(got_l))
    finally:
        dist.destroy_process_group()


def _bench_cfg4_two_ranks(tmp_path, device):
    import torch.multiprocessing as mp

    import bench
    from oracle import oracle
    oracle.build()
    n = 12                                       # graphs per rank (the 24 first graphs of the mix)
    mp.start_processes(_bench_rank_main, args=(2, _free_port(), n, str(tmp_path), device), nprocs=2, join=True,
                       start_method="spawn")
    n_total, plan = bench.cfg4_plan(n, 2)
    assert sorted(plan[0] + plan[1]) == list(range(n_total)) and plan[0] and plan[1]
    single = _solve(bench._batch_graphs(n_total, seed=1))
    assert np.array_equal(np.load(tmp_path / "counts.npy"), np.array([c for c, _ in single]))
    assert np.array_equal(np.load(tmp_path / "labels.npy"), np.concatenate([lab for _, lab in single]))


def test_bench_cfg4_sharding_on_two_gloo_ranks(tmp_path):
    """bench.py --gpus 2 --config cfg4, host side: plan, per-rank shards,
    gather in global order; the oracle stands in for the device."""
    _bench_cfg4_two_ranks(tmp_path, device=False)


@pytest.mark.gpu
def test_bench_cfg4_sharding_two_ranks_batched_engine(tmp_path):
    """The same with each rank's shard run by the batched engine (both ranks
    on device 0, independent launches): labels equal Tarjan's in order."""
    _bench_cfg4_two_ranks(tmp_path, device=True)
