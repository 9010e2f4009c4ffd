"""Benchmark of the SCC hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config cfg1|cfg2|cfg3|cfg4|cfg5] [--scale S] [--permute]

Default workload (the configuration the headline metric is quoted on):
vSlota with trim-1 and trim-2 flags (-a h -p 1 -q 1) on a seeded synthetic
R-MAT graph, scale 22 (4,194,304 vertices), edge factor 16,
(a, b, c, d) = (0.57, 0.19, 0.19, 0.05), self-loops and duplicates removed.
No public dataset is used.

One step = one complete SCC decomposition of the graph (every phase of the
driver, labels canonicalised and written).
  value : Medges/s with the CSR already resident in HBM (device pointers),
          L2 flushed (256 MiB write) before every step, CUDA events on the
          launching stream around one scc_run_async call (the whole run and
          the label write enqueued on the stream; the step ends when the
          labels are complete), max over ranks.
  e2e   : the same call through the C ABI with HOST (pinned) CSR buffers:
          the H2D copy of the forward CSR (the reverse one is built on the
          device, SCC_FLAG_DERIVE_REVERSE) and the D2H copy of the labels are
          inside the timed region; e2e.both_csr_copied times the call that
          copies both CSRs; e2e.file_to_labels times a GTgraph text file
          of the workload read, parsed and turned into both CSRs on the
          device (scc_load_graph_device), decomposed, labels back on the host.
  parity: the labels of the last timed step compared, vertex by vertex,
          with the oracle's iterative Tarjan on the same graph (checker run
          on rank 0 after the timed region).
With --gpus N > 1 every rank runs an independent replica of the graph (the
plain path does not shard); value = N * E / max-over-ranks time.  Launched
without torchrun, bench.py starts the N ranks itself (torch.distributed.run
on 127.0.0.1); under torchrun WORLD_SIZE must equal N.  --config cfg4 shards
N x 4,096 graphs over the ranks by bytes instead.

--impl reference times the reference's CPU-side answer for this path on the
host cores: the reference has no CPU SCC implementation, so this is the
project's iterative Tarjan oracle (one core, a full decomposition per step).
That arm does not load the engine's library.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "cfg1": dict(algo="g", t1=True, t2=False, warp=1,
                 desc="vHong -p 1 -q 0 on 1,024 vertices + 8,192 uniform arcs + 16 planted cycles (len 4-32)"),
    "cfg2": dict(algo="h", t1=True, t2=True, warp=1,
                 desc="vSlota -p 1 -q 1 on R-MAT scale 22, edge factor 16, (0.57,0.19,0.19,0.05), "
                      "self-loops and duplicates removed"),
    "cfg3": dict(algo="y", t1=True, t2=True, warp=8,
                 desc="wSlota -w 8 -p 1 -q 1 on a 4096x4096 grid, 70% bidirectional pairs, 30% one "
                      "random orientation, +0.1% uniform long-range arcs"),
    "cfg4": dict(algo="g", t1=True, t2=True, warp=1,
                 desc="batched: 4,096 graphs, V log-uniform in [64, 65536], mean out-degree U[4, 16], half "
                      "Erdos-Renyi, half planted-SCC chains; vHong -p 1 -q 1; one launch under a CUDA graph "
                      "vs per-graph plain launches"),
    "cfg5": dict(algo="g", t1=True, t2=True, warp=1,
                 desc="serving: Poisson arrivals at 2,000 req/s, 95% graphs from the cfg4 distribution, 5% R-MAT "
                      "scale 20 (1,048,576 vertices, edge factor 16); vHong -p 1 -q 1; 120 GB device budget; "
                      "latency = submit to labels in host memory"),
}


def _gen_graph(cfg: str, scale: int | None, device, permute: bool = False):
    from detectingscc_b200 import graphs
    if cfg == "cfg1":
        return graphs.planted_random(seed=1, device=device)
    if cfg == "cfg2":
        return graphs.rmat(scale or 22, seed=1, device=device, permute=permute)
    if cfg == "cfg3":
        return graphs.grid(scale or 4096, seed=1, device=device)
    raise ValueError(cfg)


class ClockSampler:
    """SM clock and throttle reasons sampled every ~2 ms during the timed
    region through NVML (read-only queries; the library nvidia-smi reads).
    Without NVML the record says so and holds no samples."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self.stop_ev = threading.Event()
        self.t = None
        self.max_mhz = None
        self.err = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)

            def loop():
                while not self.stop_ev.is_set():
                    try:
                        self.samples.append((pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM),
                                             pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)))
                    except Exception as e:  # pragma: no cover
                        self.err = str(e)
                        return
                    time.sleep(0.002)
            self.t = threading.Thread(target=loop, daemon=True)
            self.t.start()
        except Exception as e:
            self.err = f"nvml unavailable: {e}"

    def stop(self):
        self.stop_ev.set()
        if self.t:
            self.t.join(timeout=2)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [self.err or "no samples"], "samples": 0}
        mask = 0
        for _, r in self.samples:
            mask |= r
        reasons = sorted(k for k, bit in self.REASONS.items() if mask & bit)
        return {"sm_mhz": statistics.median(c for c, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "nvml"}


def _host_cpu():
    """CPU model and thread counts of the host the CPU baseline ran on."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        usable = os.cpu_count()
    return {"cpu_model": model, "nproc": os.cpu_count(), "usable_threads": usable}


def _config_dict(cfg_name: str, scale, V: int, E: int, world: int, permute: bool = False) -> dict:
    """The workload description both arms print (same keys and values)."""
    cfg = CONFIGS[cfg_name]
    return {"workload": f"{cfg_name}: {cfg['desc']}" + (f" [scale override {scale}]" if scale else "")
            + (", vertex ids randomly permuted (seeded, as Graph500 does)" if permute else ""),
            "V": V, "E": E, "seed": 1, "algo": cfg["algo"], "t1": cfg["t1"], "t2": cfg["t2"],
            "warp": cfg["warp"], "l2": "flushed before every step (256 MiB write)",
            "parallelism": "replicas" if world > 1 else "single GPU"}


def _peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic(cfg: str):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            t = json.load(f).get(cfg)
        return t
    except Exception:
        return None


def _dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def _max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(world: int):
    import torch
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def run_ours(args):
    import torch

    import detectingscc_b200 as scc
    from detectingscc_b200 import graphs
    world, rank, local = _dist_init()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cfg = CONFIGS[args.config]

    V, s, d = _gen_graph(args.config, args.scale, dev, args.permute)
    Fr, Fc, Br, Bc = graphs.csr_from_arcs_torch(V, s, d)
    del s, d
    E = int(Fc.shape[0])
    labels = torch.empty(V, dtype=torch.int32, device=dev)
    # pinned host copies for the end-to-end leg
    hFr, hFc, hBr, hBc = (t.cpu().pin_memory() for t in (Fr, Fc, Br, Bc))
    hlab = torch.empty(V, dtype=torch.int32).pin_memory()
    hg = scc.Graph(V, E, hFr.numpy().view(np.uint32), hFc.numpy().view(np.uint32), hBr.numpy().view(np.uint32),
                   hBc.numpy().view(np.uint32))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)

    eng = scc.Engine(local)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    def step_dev(instrument=False, wait=True):
        return eng.run_device(V, E, Fr, Fc, Br, Bc, labels_out=labels, algo=cfg["algo"], t1=cfg["t1"],
                              t2=cfg["t2"], warp=cfg["warp"], stream=sh, instrument=instrument, wait=wait)

    # warm-up
    for _ in range(args.warmup):
        step_dev()
    # work counters for the roofline (separate, instrumented, untimed run)
    ins = step_dev(instrument=True).stats

    clocks = ClockSampler(local)
    _barrier(world)
    clocks.start()
    step_ms, kern_ms, launches = [], [], 0
    res = None
    for _ in range(args.steps):
        flush.zero_()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        step_dev(wait=False)          # enqueued on the stream; the step ends with the labels written
        ev1.record(stream)
        ev1.synchronize()
        res = eng.finish()            # counters and kernel time of the step (after the timed window)
        step_ms.append(ev0.elapsed_time(ev1))
        kern_ms.append(res.stats["kernel_ms"])
        launches += res.stats["gpu_launches"]
    _barrier(world)
    clk = clocks.stop()
    t_step = _max_over_ranks(sum(step_ms) / len(step_ms), world)
    t_kern = _max_over_ranks(sum(kern_ms) / len(kern_ms), world)

    # end-to-end: host pinned CSR in, labels out, through the C ABI; twice:
    # both CSRs copied (the reference's interface), and only the forward CSR
    # copied with the reverse one built on the device (SCC_FLAG_DERIVE_REVERSE)
    hlab_np = hlab.numpy().view(np.uint32)

    def e2e_leg(derive):
        for _ in range(max(1, args.warmup)):
            eng.run(hg, algo=cfg["algo"], t1=cfg["t1"], t2=cfg["t2"], warp=cfg["warp"], out=hlab_np,
                    derive_reverse=derive)
        _barrier(world)
        ms = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            r = eng.run(hg, algo=cfg["algo"], t1=cfg["t1"], t2=cfg["t2"], warp=cfg["warp"], out=hlab_np,
                        derive_reverse=derive)
            ms.append((time.perf_counter() - t0) * 1e3)
        _barrier(world)
        assert r.num_sccs == res.num_sccs
        return _max_over_ranks(sum(ms) / len(ms), world), r.labels.copy()

    t_e2e_both, lab_both = e2e_leg(False)
    t_e2e, lab_fwd = e2e_leg(True)
    assert np.array_equal(lab_both, lab_fwd)
    assert np.array_equal(lab_fwd, labels.cpu().numpy().view(np.uint32))
    file_leg = None if args.no_file_leg else file_to_labels(eng, hg, labels, lab_fwd, cfg, sh, world, rank, args)

    B_alg = 8 * ins["edges_scanned"] + 12 * ins["vertex_visits"]
    peak, peak_kind = _peak_hbm()
    achieved = B_alg / (t_kern * 1e-3) / 1e9
    tr = _traffic(args.config if args.scale is None else None)
    out = {
        "metric": f"SCC Medges/s ({'vSlota' if cfg['algo'] == 'h' else cfg['algo']}, {args.config})",
        "value": round(world * E / (t_step * 1e-3) / 1e6, 2),
        "unit": "Medges/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(t_step, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded generator, no dataset)",
        "config": _config_dict(args.config, args.scale, V, E, world, args.permute),
        "num_sccs": int(res.num_sccs),
        "counts": {"trim1": int(res.num_trim1), "trim2": int(res.num_trim2), "pivot": int(res.num_pivot)},
        "passes": res.stats["passes"], "outer_iters": res.stats["outer_iters"],
        "kernel_ms": round(t_kern, 4),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": tr.get("dram_bytes_per_launch") if tr else None,
                     "B_alg": int(B_alg), "T_e": int(ins["edges_scanned"]), "T_v": int(ins["vertex_visits"]),
                     "T_e_over_E": round(ins["edges_scanned"] / max(E, 1), 3),
                     "T_v_over_V": round(ins["vertex_visits"] / max(V, 1), 3),
                     "B_floor_GBps": round((8 * E + 12 * V) / (t_kern * 1e-3) / 1e9, 1),
                     "kernel": "k_scc_block (the whole driver on one CTA)" if res.stats.get("used_block_path")
                     else "k_scc_grid (persistent cooperative SCC kernel)"},
        "e2e": {"value": round(world * E / (t_e2e * 1e-3) / 1e6, 2), "unit": "Medges/s",
                "ms_per_step": round(t_e2e, 3),
                "h2d_bytes_per_step": int(4 * ((V + 2) + E)),
                "d2h_bytes_per_step": int(4 * V + 512),
                "path": "forward CSR from pinned host memory, reverse CSR built on the device "
                        "(SCC_FLAG_DERIVE_REVERSE), labels back to pinned host memory",
                "both_csr_copied": {"value": round(world * E / (t_e2e_both * 1e-3) / 1e6, 2),
                                    "ms_per_step": round(t_e2e_both, 3),
                                    "h2d_bytes_per_step": int(4 * (2 * (V + 2) + 2 * E))}},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if file_leg:
        out["e2e"]["file_to_labels"] = file_leg
    if rank == 0:
        # checker and CPU baseline (after the timed region): the oracle's
        # iterative Tarjan on the same host CSR
        from oracle import oracle
        if not args.no_parity:
            ref_lab, ref_n = oracle.tarjan(V, hg.Fr, hg.Fc)
            got = labels.cpu().numpy().view(np.uint32)
            nbad = int(np.count_nonzero(got != ref_lab[1:]))
            out["parity"] = nbad == 0 and int(res.num_sccs) == ref_n
            out["parity_detail"] = {"against": "oracle iterative Tarjan (canonical min-id labels)",
                                    "labels_checked": V, "labels_differing": nbad, "num_sccs_oracle": ref_n,
                                    "labels_of": "last timed step; the e2e legs' labels equal them"}
        if world == 1 and not args.no_cpu_baseline:
            t_cpu, reps = oracle.time_tarjan(V, hg.Fr, hg.Fc, budget_s=20.0, max_reps=3)
            out["cpu_baseline"] = {"value": round(E / t_cpu / 1e6, 2), "unit": "Medges/s", "cores": 1,
                                   "kind": "port", "sample": f"full graph, iterative Tarjan, median of {reps} "
                                                             f"run(s), {t_cpu:.2f} s per run",
                                   "host": _host_cpu()}
        print(json.dumps(out), flush=True)
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def file_to_labels(eng, hg, labels, expect, cfg, sh, world, rank, args):
    """The workload as a GTgraph text file (written once by the library's
    writer, untimed), then timed: scc_load_graph_device (file read, text
    parsed and both CSRs built on the device), the SCC run, labels copied to
    the host.  The file is read from the page cache."""
    import tempfile

    import torch

    import detectingscc_b200 as scc
    path = os.path.join(tempfile.gettempdir(), f"sccb_bench_{os.getpid()}_{rank}.gr")
    try:
        scc.save_gtgraph(path, hg)
        nbytes = os.path.getsize(path)
        ms, got = [], None
        for i in range(1 + max(1, min(args.steps, 3))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            V, E, Fr, Fc, Br, Bc = eng.load_graph_device(path, stream=sh)
            eng.run_device(V, E, Fr, Fc, Br, Bc, labels_out=labels, algo=cfg["algo"], t1=cfg["t1"], t2=cfg["t2"],
                           warp=cfg["warp"], stream=sh)
            got = labels.cpu()
            if i:
                ms.append((time.perf_counter() - t0) * 1e3)
        assert np.array_equal(got.numpy().view(np.uint32), expect)   # the same labels as the in-memory legs
        t = _max_over_ranks(sum(ms) / len(ms), world)
        return {"value": round(world * hg.E / (t * 1e-3) / 1e6, 2), "unit": "Medges/s", "ms_per_step": round(t, 2),
                "file_bytes": int(nbytes), "reps": len(ms),
                "path": "GTgraph text file -> scc_load_graph_device (host read, device parse, radix-sorted CSRs) "
                        "-> SCC -> labels in host memory"}
    finally:
        if os.path.exists(path):
            os.remove(path)


def _pinned_graph(g):
    """The graph's CSR arrays copied into page-locked host memory."""
    import torch

    import detectingscc_b200 as scc
    arrs = [torch.from_numpy(a.view(np.int32)).pin_memory() for a in (g.Fr, g.Fc, g.Br, g.Bc)]
    h = scc.Graph(g.V, g.E, *(t.numpy().view(np.uint32) for t in arrs))
    h._pins = arrs
    return h


def _batch_graphs(n_graphs: int, seed: int = 1, indices=None):
    """Graphs `indices` (default all n_graphs) of the seeded mix, built on a thread pool."""
    import concurrent.futures as cf

    import detectingscc_b200 as scc
    from detectingscc_b200 import graphs
    idx = list(range(n_graphs)) if indices is None else list(indices)
    with cf.ThreadPoolExecutor(os.cpu_count() or 1) as ex:   # the CSR builder releases the GIL
        return list(ex.map(lambda i: scc.graph_from_arcs(*graphs.batch_mix_graph(i, seed=seed)), idx))


def cfg4_plan(n_graphs: int, world: int):
    """cfg4 on `world` ranks: world x n_graphs graphs of the mix (seed 1),
    split over the ranks by CSR bytes (greedy longest-processing-time; every
    rank computes the same plan from the sizes alone).  Returns (total
    graphs, plan) with plan[r] the global indices rank r builds and runs."""
    from detectingscc_b200 import graphs
    from detectingscc_b200.shard import shard_by_bytes
    n_total = n_graphs * world
    sizes = [graphs.batch_mix_bytes(V, deg) for V, deg in graphs.batch_mix_sizes(n_total, seed=1)]
    return n_total, shard_by_bytes(sizes, world)


def run_batch(args):
    """cfg4: graphs/s of the batched launch vs per-graph plain launches."""
    import torch

    import detectingscc_b200 as scc
    world, rank, local = _dist_init()
    torch.cuda.set_device(local)
    cfg = CONFIGS["cfg4"]
    from detectingscc_b200.shard import gather_in_order
    # world x 4096 graphs, sharded by bytes (greedy LPT); each rank builds and runs its own shard
    n_total, plan = cfg4_plan(args.scale or 4096, world)
    gs = _batch_graphs(n_total, seed=1, indices=plan[rank])
    eng = scc.Engine(local)
    b = scc.Batch(eng, gs)
    t_ins = time.perf_counter()
    best_t, best_q, _ = b.autotune(algo=cfg["algo"], t1=cfg["t1"], t2=cfg["t2"], warp=cfg["warp"])
    best_c, best_big, n_cl = b.cluster()
    t_tune = time.perf_counter() - t_ins
    for _ in range(args.warmup):
        b.run(algo=cfg["algo"], t1=cfg["t1"], t2=cfg["t2"], warp=cfg["warp"], labels=False)
    clocks = ClockSampler(local)
    _barrier(world)
    clocks.start()
    ms = []
    for _ in range(args.steps):
        _, res, st = b.run(algo=cfg["algo"], t1=cfg["t1"], t2=cfg["t2"], warp=cfg["warp"], labels=False)
        ms.append(st["kernel_ms"])
    _barrier(world)
    clk = clocks.stop()
    t_batch = _max_over_ranks(sum(ms) / len(ms), world)
    # per-graph plain launches of the same engine (sequential, state resident)
    seq = []
    for _ in range(max(1, min(3, args.steps))):
        _, res_s, st_s = b.run(algo=cfg["algo"], t1=cfg["t1"], t2=cfg["t2"], warp=cfg["warp"], labels=False,
                               sequential=True)
        seq.append(st_s["kernel_ms"])
    t_seq = _max_over_ranks(sum(seq) / len(seq), world)
    assert [r[0] for r in res] == [r[0] for r in res_s]
    # per-graph SCC counts back on rank 0 in global order (host-side gather, no data-path collective)
    counts = gather_in_order([r[0] for r in res], plan, rank, dst=0)
    assert rank != 0 or (len(counts) == n_total and None not in counts)
    # end to end: upload every graph from (page-locked) host memory, run, read all labels back
    import torch as _t
    pins = [_pinned_graph(g) for g in gs]
    hlab = _t.zeros(b.total_vertices, dtype=_t.int32).pin_memory().numpy().view(np.uint32)
    e2e = []
    for _ in range(max(1, min(3, args.steps))):
        t0 = time.perf_counter()
        b2 = scc.Batch(eng, pins)
        b2.set_schedule(best_t, best_q)
        b2.set_cluster(best_c, best_big)
        b2.run(algo=cfg["algo"], t1=cfg["t1"], t2=cfg["t2"], warp=cfg["warp"], out=hlab)
        e2e.append(time.perf_counter() - t0)
        b2.close()
    t_e2e = _max_over_ranks(sum(e2e) / len(e2e), world)
    sumE = b.total_edges
    out = {
        "metric": "batched SCC graphs/s (cfg4)", "value": round(n_total / (t_batch * 1e-3), 1),
        "unit": "graphs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t_batch, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": f"cfg4: {cfg['desc']}", "graphs": n_total, "graphs_this_rank": len(gs),
                   "sum_V_this_rank": b.total_vertices, "sum_E_this_rank": sumE, "seed": 1, "schedule": {"threads": best_t, "qcap": best_q, "cluster": best_c,
                                                          "big_vertices": best_big, "cluster_graphs": n_cl,
                                                          "autotune_s": round(t_tune, 2)},
                   "l2": "inputs larger than L2",
                   "parallelism": f"{n_total} graphs sharded over {world} ranks by bytes (greedy LPT)" if world > 1
                   else "single GPU"},
        "per_graph_plain": {"ms_per_batch": round(t_seq, 3), "graphs_per_s": round(n_total / (t_seq * 1e-3), 1)},
        "batched_over_plain": round(t_seq / t_batch, 2),
        "Medges_per_s": round(world * sumE / (t_batch * 1e-3) / 1e6, 1),
        "e2e": {"value": round(n_total / t_e2e, 1), "unit": "graphs/s", "ms_per_step": round(t_e2e * 1e3, 2),
                "h2d_bytes_per_step": int(sum(g.nbytes for g in gs)), "d2h_bytes_per_step": int(4 * b.total_vertices)},
        "gpu_launches": int(args.steps), "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import concurrent.futures as cf

        from oracle import oracle
        cores = os.cpu_count() or 1
        sample = gs[: max(64, len(gs) // 8)]
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(cores) as ex:
            list(ex.map(lambda g: oracle.tarjan(g.V, g.Fr, g.Fc), sample))
        t_cpu = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(len(sample) / t_cpu, 1), "unit": "graphs/s", "cores": cores,
                               "kind": "port", "sample": f"first {len(sample)} graphs of the mix, iterative "
                                                         f"Tarjan per graph on a {cores}-thread pool",
                               "host": _host_cpu()}
    if rank == 0:
        print(json.dumps(out), flush=True)
    b.close()
    eng.close()


def run_serve(args):
    """cfg5: p50 / p99 latency and graphs/s of the request server."""
    import threading

    import torch

    import detectingscc_b200 as scc
    from detectingscc_b200 import graphs
    world, rank, local = _dist_init()
    torch.cuda.set_device(local)
    cfg = CONFIGS["cfg5"]
    rate = 2000.0
    duration = float(args.scale or max(args.steps, 30))
    rng = np.random.default_rng(7 + rank)

    small = [_pinned_graph(g) for g in _batch_graphs(512, seed=11 + rank)]   # one request stream per rank
    large = []
    for k in range(4):
        V, s_, d_ = graphs.rmat(20, seed=100 + k + 10 * rank, device=torch.device("cuda", local))
        large.append(_pinned_graph(graphs.to_graph(V, s_, d_)))
    pool = small + large
    # solo answers for the in-mix check
    eng = scc.Engine(local)
    solo = [eng.run(g, algo=cfg["algo"], t1=cfg["t1"], t2=cfg["t2"]).labels.copy() for g in pool]
    eng.close()
    srv = scc.Server(local, algo=cfg["algo"], t1=cfg["t1"], t2=cfg["t2"], budget_bytes=120 * 10**9)
    # warm-up: every large graph and a burst of small ones
    for _ in range(max(args.warmup, 1)):
        for g in large + small[:64]:
            srv.submit(g)
        got = 0
        while got < len(large) + 64:
            got += len(srv.poll(256, wait_ms=100))
    lat_s, lat_l, qms, done, checked, bad, edges, h2d, d2h = [], [], [], 0, 0, 0, 0, 0, 0
    pool_of = {}
    lock = threading.Lock()
    stop = threading.Event()
    sent = [0]

    def producer():
        t_next = time.perf_counter()
        t_end = t_next + duration
        while True:
            t_next += rng.exponential(1.0 / rate)
            if t_next > t_end:
                break
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            i = len(small) + int(rng.integers(len(large))) if rng.random() < 0.05 else int(rng.integers(len(small)))
            with lock:   # a fast request can be polled before submit() returns here
                pool_of[srv.submit(pool[i])] = i
            sent[0] += 1
        stop.set()

    launches0 = srv.launches()
    clocks = ClockSampler(local)
    clocks.start()
    th = threading.Thread(target=producer, daemon=True)
    t0 = time.perf_counter()
    th.start()
    while not (stop.is_set() and done >= sent[0]):
        for r in srv.poll(1024, wait_ms=20):
            with lock:
                i = pool_of.pop(r["ticket"])
            done += 1
            if r["status"] != 0:
                bad += 1
                continue
            (lat_l if i >= len(small) else lat_s).append(r["latency_ms"])
            qms.append(r["queue_ms"])
            g = pool[i]
            edges += g.E
            h2d += g.nbytes
            d2h += 4 * g.V
            if done % 17 == 0 or i >= len(small):   # bit-exact check against the solo run
                checked += 1
                bad += int(not np.array_equal(r["labels"], solo[i]))
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    info = srv.info()
    launches = srv.launches() - launches0
    srv.close()
    lat = np.array(lat_s + lat_l)
    pct = lambda a, q: round(float(np.percentile(a, q)), 3) if len(a) else None  # noqa: E731
    out = {
        "metric": "serving SCC p99 latency (cfg5)", "value": pct(lat, 99), "unit": "ms",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": f"cfg5: {cfg['desc']}", "duration_s": duration, "rate_req_per_s": rate,
                   "pool": {"small_graphs": len(small), "large_graphs": len(large)},
                   "server": {"lanes": 8, "batch_threads": 1024, "qcap": 256, "cluster": 4, "big_vertices": 16384,
                              "large_cluster": 16},
                   "inputs": "page-locked host CSR per request, labels to pageable host arrays",
                   "parallelism": "one server per rank" if world > 1 else "single GPU"},
        "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "p50_queue_ms": pct(qms, 50),
        "small": {"p50_ms": pct(lat_s, 50), "p99_ms": pct(lat_s, 99), "n": len(lat_s)},
        "large": {"p50_ms": pct(lat_l, 50), "p99_ms": pct(lat_l, 99), "n": len(lat_l)},
        "graphs_per_s": round(done / wall, 1), "Medges_per_s": round(edges / wall / 1e6, 1),
        "requests": int(done), "failed_or_mismatched": int(bad), "checked_bit_exact": int(checked),
        "server_info": info,
        "e2e": {"value": round(done / wall, 1), "unit": "graphs/s", "step": "one request",
                "h2d_bytes_per_step": int(h2d / max(done, 1)), "d2h_bytes_per_step": int(d2h / max(done, 1))},
        "gpu_launches": int(launches), "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_reference(args):
    world, rank, local = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), \
        int(os.environ.get("LOCAL_RANK", "0"))
    if rank != 0:
        return
    import torch

    from detectingscc_b200 import graphs   # the seeded generators (PyTorch only; the engine is not loaded)
    from oracle import oracle
    from oracle.gtgraph_ref import build_csr
    cfg = CONFIGS[args.config]
    if args.config in ("cfg4", "cfg5"):
        # both are many independent graphs of the cfg4 mix: Tarjan per graph on all host cores
        import concurrent.futures as cf
        from types import SimpleNamespace

        def mk(i):
            V, s_, d_ = graphs.batch_mix_graph(i, seed=1)
            Fr, Fc, _, _ = build_csr(V, s_, d_)
            return SimpleNamespace(V=V, Fr=Fr, Fc=Fc)
        with cf.ThreadPoolExecutor(os.cpu_count() or 1) as ex:
            gs = list(ex.map(mk, range(args.scale or 4096)))
        cores = os.cpu_count() or 1
        sample = gs[: max(64, len(gs) // 8)]
        times = []
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            with cf.ThreadPoolExecutor(cores) as ex:
                list(ex.map(lambda g: oracle.tarjan(g.V, g.Fr, g.Fc), sample))
            if i >= args.warmup:
                times.append(time.perf_counter() - t0)
        v = round(len(sample) / (sum(times) / len(times)), 1)
        metric = "batched SCC graphs/s (cfg4)" if args.config == "cfg4" else "serving SCC graphs/s (cfg5, CPU throughput)"
        print(json.dumps({"impl": "reference", "metric": metric, "value": v, "unit": "graphs/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
                          "config": {"workload": f"{args.config}: {cfg['desc']}", "graphs": len(gs)},
                          "cpu_baseline": {"value": v, "unit": "graphs/s", "cores": cores, "kind": "port",
                                           "sample": f"first {len(sample)} graphs per step, Tarjan per graph on a "
                                                     f"{cores}-thread pool (the reference has no CPU SCC path)",
                                           "host": _host_cpu()},
                          "e2e": {"value": v, "unit": "graphs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    dev = torch.device("cuda", local) if torch.cuda.is_available() else torch.device("cpu")
    V, s, d = _gen_graph(args.config, args.scale, dev, args.permute)
    Fr, Fc, Br, Bc = (t.cpu().numpy().view(np.uint32) for t in graphs.csr_from_arcs_torch(V, s, d))
    E = int(Fc.shape[0])
    for _ in range(args.warmup):
        oracle.tarjan(V, Fr, Fc)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.tarjan(V, Fr, Fc)
        times.append(time.perf_counter() - t0)
    t = sum(times) / len(times)
    v = round(E / t / 1e6, 2)
    out = {
        "impl": "reference",
        "metric": f"SCC Medges/s ({'vSlota' if cfg['algo'] == 'h' else cfg['algo']}, {args.config})",
        "value": v, "unit": "Medges/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t * 1e3, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (seeded generator, no dataset)",
        "config": _config_dict(args.config, args.scale, V, E, world, args.permute),
        "cpu_baseline": {"value": v, "unit": "Medges/s", "cores": 1, "kind": "port",
                         "sample": "full graph per step; the reference has no CPU SCC path, so this is the "
                                   "project's iterative Tarjan oracle on one host core", "host": _host_cpu()},
        "e2e": {"value": v, "unit": "Medges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    ref_gpu = _reference_gpu_time(args, V, E, Fr, Fc, Br, Bc, cfg)
    if ref_gpu:
        out["reference_gpu"] = ref_gpu
    print(json.dumps(out), flush=True)


def _reference_gpu_time(args, V, E, Fr, Fc, Br, Bc, cfg):
    """The reference's own CUDA drivers (oracle/_ref/scc_ref, built from its
    unchanged sources) on the same graph: its printed count and its own
    "Time :" (which includes its cudaMalloc and host-to-device copies)."""
    import re
    import tempfile

    ref = os.path.join(ROOT, "oracle", "_ref", "scc_ref")
    if not os.path.exists(ref):
        return None
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "graph.bin")
        # the binary CSR both loaders read: "SCCBIN01", u64 V, u64 E, Fr, Fc, Br, Bc (u32)
        with open(path, "wb") as f:
            f.write(b"SCCBIN01")
            f.write(np.array([V, E], dtype=np.uint64).tobytes())
            for a in (Fr, Fc, Br, Bc):
                f.write(np.ascontiguousarray(a, dtype=np.uint32).tobytes())
        runs = []
        for _ in range(3):
            try:
                r = subprocess.run([ref, "-a", cfg["algo"], "-p", "1" if cfg["t1"] else "0",
                                    "-q", "1" if cfg["t2"] else "0", "-w", str(cfg["warp"]), "-f", path],
                                   capture_output=True, text=True, timeout=300)
            except subprocess.TimeoutExpired:
                return {"unavailable": "reference binary exceeded 300 s"}
            t = re.search(r"Time : ([0-9.]+)", r.stdout)
            n = re.search(r"Number Of Sccs : (-?\d+)", r.stdout)
            if r.returncode != 0 or not t:
                return {"unavailable": f"reference binary exit {r.returncode}"}
            runs.append((float(t.group(1)), int(n.group(1)) if n else None))
    best = min(runs)
    return {"time_ms": best[0], "num_sccs": best[1], "Medges_per_s": round(E / (best[0] * 1e-3) / 1e6, 2),
            "note": "reference CUDA drivers built from their sources for sm_100a; Time includes their "
                    "cudaMalloc + H2D; best of 3"}


def _launch_ranks(n: int) -> int:
    """Starts n ranks of this same command (torch.distributed.run on
    127.0.0.1, one process per GPU) and returns their exit status."""
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg2", choices=sorted(CONFIGS))
    ap.add_argument("--scale", type=int, default=None, help="smaller graph (profiling aid, not a bench value)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the label check against the oracle")
    ap.add_argument("--permute", action="store_true", help="cfg2 with its vertex ids randomly permuted")
    ap.add_argument("--no-file-leg", action="store_true", help="skip the GTgraph file-to-labels measurement")
    args = ap.parse_args()
    world = os.environ.get("WORLD_SIZE")
    if world is None and args.gpus > 1:
        sys.exit(_launch_ranks(args.gpus))
    if world is not None and int(world) != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch one rank per GPU", file=sys.stderr)
        sys.exit(2)
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "cfg4":
        run_batch(args)
    elif args.config == "cfg5":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
