"""Python host mirror of the reference's interface on top of the C ABI.

Reference surface (same names, argument meaning and behaviour):

* ``loadFullGraph(filename)``                       load.h:6, load.cpp:12-140
* ``vHong(CSize, RSize, Fc, Fr, Bc, Br, t1, t2)``     scc.h:52, scc_WCC.cu:573
* ``vSlota(CSize, RSize, Fc, Fr, Bc, Br, t1, t2)``    scc.h:50, scc_Coloring.cu:403
* ``wHong(..., t1, t2, warpSize)``                  scc.h:51, scc_WCC.cu:53
* ``wSlota(..., t1, t2, warpSize)``                 scc.h:49, scc_Coloring.cu:6

The drivers print exactly what the reference prints (through the native
library's stdout) and return the SCC count.  ``Engine`` adds what the
reference never exposed: per-vertex canonical labels, device-resident
inputs, counters and timings.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _native as N

ALGOS = {"g": "vHong", "h": "vSlota", "x": "wHong", "y": "wSlota"}


@dataclass
class Graph:
    """Host CSR in the reference layout (1-based; Fr/Br have V+2 entries)."""
    V: int
    E: int
    Fr: np.ndarray
    Fc: np.ndarray
    Br: np.ndarray
    Bc: np.ndarray
    name: str = ""

    def __post_init__(self):
        for k in ("Fr", "Fc", "Br", "Bc"):
            a = np.ascontiguousarray(getattr(self, k), dtype=np.uint32)
            setattr(self, k, a)

    @property
    def nbytes(self) -> int:
        return 4 * (2 * (self.V + 2) + 2 * self.E)


@dataclass
class Result:
    labels: Optional[np.ndarray]      # V entries, labels[i] = min id of SCC of vertex i+1
    num_sccs: int
    num_trim1: int
    num_trim2: int
    num_pivot: int
    stats: dict = field(default_factory=dict)


def _ptr(a) -> int:
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return int(a)


def _algo_code(algo) -> int:
    if isinstance(algo, str):
        if algo in ALGOS:
            return ord(algo)
        inv = {v: k for k, v in ALGOS.items()}
        if algo in inv:
            return ord(inv[algo])
        raise ValueError(f"unknown algorithm {algo!r}")
    return int(algo)


class Engine:
    """An scc_context on one CUDA device."""

    def __init__(self, device: int = 0):
        self._lib = N.lib()
        h = ctypes.c_void_p()
        N.check(self._lib.scc_create(int(device), ctypes.byref(h)), "scc_create")
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            self._lib.scc_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown ordering
        try:
            self.close()
        except Exception:
            pass

    def set_tuning(self, key: str, value: int) -> None:
        N.check(self._lib.scc_set_tuning(self._h, key.encode(), int(value)), f"scc_set_tuning({key})")

    PHASES = {1: "init", 2: "trim1_once", 3: "trim1_apply", 4: "trim1_fix", 5: "trim2", 6: "trim2_apply",
              7: "first_pivot", 8: "bfs0", 9: "bfs", 10: "prop", 11: "hong_update", 12: "slota_first_update",
              13: "slota_peel_update", 14: "rename", 15: "pivots", 16: "bfs_pull", 17: "prop_pull",
              18: "res_tag", 19: "res_extract", 20: "res_solve"}

    def trace(self):
        """Per-pass (phase, microseconds, items pushed) of the last run (needs set_tuning('trace', n))."""
        n = ctypes.c_uint32(0)
        t0 = ctypes.c_uint64(0)
        N.check(self._lib.scc_get_trace(self._h, None, 0, ctypes.byref(n), ctypes.byref(t0)))
        buf = (ctypes.c_uint64 * (2 * max(n.value, 1)))()
        N.check(self._lib.scc_get_trace(self._h, buf, n.value, ctypes.byref(n), ctypes.byref(t0)))
        out, prev = [], t0.value
        for i in range(n.value):
            t, info = buf[2 * i], buf[2 * i + 1]
            out.append((self.PHASES.get(info & 0xFF, str(info & 0xFF)), (t - prev) / 1e3, info >> 8))
            prev = t
        return out

    def run(self, g: Graph, algo="h", t1=True, t2=True, warp=1, labels=True,
            instrument=False, force=None, out: Optional[np.ndarray] = None,
            derive_reverse: bool = False) -> Result:
        """Run on a host graph: the call copies the CSR in and the labels out.

        out: optional preallocated host array (e.g. pinned) of V uint32.
        derive_reverse: copy only the forward CSR and build the reverse one on
        the device (g.Br / g.Bc are not read).
        """
        flags = (N.FLAG_TRIM1 if t1 else 0) | (N.FLAG_TRIM2 if t2 else 0)
        flags |= N.FLAG_INSTRUMENT if instrument else 0
        flags |= N.FLAG_DERIVE_REVERSE if derive_reverse else 0
        if force == "grid":
            flags |= N.FLAG_FORCE_GRID
        elif force == "block":
            flags |= N.FLAG_FORCE_BLOCK
        view = N.CsrView(g.V, g.E, _ptr(g.Fr), _ptr(g.Fc), _ptr(g.Br), _ptr(g.Bc))
        if labels and out is None:
            out = np.zeros(max(g.V, 1), dtype=np.uint32)
        elif not labels:
            out = None
        st = N.Stats()
        rc = self._lib.scc_run(self._h, ctypes.byref(view), _algo_code(algo), flags, int(warp),
                               _ptr(out), ctypes.byref(st), None)
        N.check(rc, f"scc_run (device error location {st.error_where})" if rc else "scc_run")
        return Result(out[:g.V] if labels else None, st.num_sccs, st.num_trim1, st.num_trim2,
                      st.num_pivot, st.as_dict())

    def detect(self, g: Graph, Pr=None, t1=True, t2=True) -> dict:
        """detectSCC (-a d, scc_WCC.cu:1000-1617) on a host graph with METIS
        partition ids Pr (V+2 entries, Pr[v] for vertex v; None: one partition).
        Returns the reference's printed count and its parts."""
        P = np.zeros(g.V + 2, dtype=np.uint32) if Pr is None else np.ascontiguousarray(Pr, dtype=np.uint32)
        if P.shape[0] < g.V + 2:
            raise ValueError("Pr needs V + 2 entries")
        view = N.CsrView(g.V, g.E, _ptr(g.Fr), _ptr(g.Fc), _ptr(g.Br), _ptr(g.Bc))
        r = N.DetectResult()
        flags = (N.FLAG_TRIM1 if t1 else 0) | (N.FLAG_TRIM2 if t2 else 0)
        N.check(self._lib.scc_detect(self._h, ctypes.byref(view), _ptr(P), flags, ctypes.byref(r)), "scc_detect")
        return {k: getattr(r, k) for k, _ in N.DetectResult._fields_}

    def load_graph_device(self, path: str, stream=None):
        """Parse a GTgraph file (or the binary CSR format) on the device and build
        both CSRs there.  Returns (V, E, Fr, Fc, Br, Bc) with device pointers
        (ints) into this engine's CSR arrays, for run_device; they stay valid
        until the next load or run with host inputs on this engine."""
        view = N.CsrView()
        N.check(self._lib.scc_load_graph_device(self._h, path.encode(), ctypes.byref(view), stream),
                f"scc_load_graph_device({path})")
        return view.num_vertices, view.num_edges, view.Fr, view.Fc, view.Br, view.Bc

    def derive_reverse(self, V: int, E: int, Fr, Fc, Br, Bc, stream=None) -> None:
        """Fill device arrays Br (V+2) and Bc (E) with the reverse CSR of (Fr, Fc)."""
        if stream is None and hasattr(Fr, "device") and getattr(Fr.device, "type", "") == "cuda":
            import torch
            stream = torch.cuda.current_stream(Fr.device).cuda_stream
        N.check(self._lib.scc_derive_reverse(self._h, _ptr(Fr), _ptr(Fc), int(V), int(E), _ptr(Br), _ptr(Bc), stream),
                "scc_derive_reverse")

    def run_device(self, V: int, E: int, Fr, Fc, Br, Bc, labels_out=None, algo="h", t1=True, t2=True,
                   warp=1, instrument=False, stream=None, force=None, derive_reverse: bool = False,
                   wait: bool = True) -> Optional[Result]:
        """Run on device-resident CSR (torch CUDA tensors or raw device pointers).

        labels_out: device buffer of V uint32/int32 entries, or None.
        stream: a cudaStream_t handle (int); None means the current PyTorch stream
                of the tensors' device (or the legacy default stream for raw pointers).
        wait: False enqueues the run and returns None at once (scc_run_async);
              labels_out is complete in the stream's order and finish() returns
              the Result.
        """
        flags = N.FLAG_DEVICE | (N.FLAG_TRIM1 if t1 else 0) | (N.FLAG_TRIM2 if t2 else 0)
        flags |= N.FLAG_INSTRUMENT if instrument else 0
        flags |= N.FLAG_DERIVE_REVERSE if derive_reverse else 0
        if force == "grid":
            flags |= N.FLAG_FORCE_GRID
        elif force == "block":
            flags |= N.FLAG_FORCE_BLOCK
        if stream is None and hasattr(Fr, "device") and getattr(Fr.device, "type", "") == "cuda":
            # order after the producer of the tensors: run on their device's current stream
            import torch
            stream = torch.cuda.current_stream(Fr.device).cuda_stream
        view = N.CsrView(int(V), int(E), _ptr(Fr), _ptr(Fc), _ptr(Br), _ptr(Bc))
        if not wait:
            N.check(self._lib.scc_run_async(self._h, ctypes.byref(view), _algo_code(algo), flags, int(warp),
                                            _ptr(labels_out), stream), "scc_run_async")
            return None
        st = N.Stats()
        rc = self._lib.scc_run(self._h, ctypes.byref(view), _algo_code(algo), flags, int(warp),
                               _ptr(labels_out), ctypes.byref(st), stream)
        N.check(rc, f"scc_run (device error location {st.error_where})" if rc else "scc_run")
        return Result(None, st.num_sccs, st.num_trim1, st.num_trim2, st.num_pivot, st.as_dict())

    def finish(self) -> Result:
        """Waits for the last run_device(..., wait=False) and returns its Result."""
        st = N.Stats()
        rc = self._lib.scc_finish(self._h, ctypes.byref(st))
        N.check(rc, f"scc_finish (device error location {st.error_where})" if rc else "scc_finish")
        return Result(None, st.num_sccs, st.num_trim1, st.num_trim2, st.num_pivot, st.as_dict())


class Batch:
    """Many independent graphs resident on one device, run in one launch."""

    def __init__(self, engine: "Engine", graphs):
        self._lib = engine._lib
        self.engine = engine
        self.graphs = list(graphs)
        self._keep = self.graphs  # host arrays must outlive the upload only; kept for offsets
        views = (N.CsrView * max(len(self.graphs), 1))()
        for i, g in enumerate(self.graphs):
            views[i] = N.CsrView(g.V, g.E, _ptr(g.Fr), _ptr(g.Fc), _ptr(g.Br), _ptr(g.Bc))
        h = ctypes.c_void_p()
        N.check(self._lib.scc_batch_create(engine._h, views, len(self.graphs), ctypes.byref(h)), "scc_batch_create")
        self._h = h
        self.offsets = np.concatenate([[0], np.cumsum([g.V for g in self.graphs])]).astype(np.int64)
        self.total_vertices = int(self.offsets[-1])
        self.total_edges = int(sum(g.E for g in self.graphs))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.scc_batch_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def set_schedule(self, threads: int, qcap: int) -> None:
        N.check(self._lib.scc_batch_set_schedule(self._h, int(threads), int(qcap)), "scc_batch_set_schedule")

    def schedule(self):
        t, q = ctypes.c_int(0), ctypes.c_uint32(0)
        N.check(self._lib.scc_batch_get_schedule(self._h, ctypes.byref(t), ctypes.byref(q)))
        return t.value, q.value

    def set_cluster(self, cluster: int, big_vertices: int = 16384) -> None:
        """Run graphs with at least big_vertices vertices on clusters of `cluster` CTAs (1: off)."""
        N.check(self._lib.scc_batch_set_cluster(self._h, int(cluster), int(big_vertices)), "scc_batch_set_cluster")

    def cluster(self):
        """(cluster size, big_vertices, number of graphs that run on whole clusters)."""
        c, b, n = ctypes.c_int(0), ctypes.c_uint32(0), ctypes.c_uint32(0)
        N.check(self._lib.scc_batch_get_cluster(self._h, ctypes.byref(c), ctypes.byref(b), ctypes.byref(n)))
        return c.value, b.value, n.value

    def autotune(self, algo="h", t1=True, t2=True, warp=1):
        t, q, ms = ctypes.c_int(0), ctypes.c_uint32(0), ctypes.c_float(0)
        flags = (N.FLAG_TRIM1 if t1 else 0) | (N.FLAG_TRIM2 if t2 else 0)
        N.check(self._lib.scc_batch_autotune(self._h, _algo_code(algo), flags, int(warp), ctypes.byref(t),
                                             ctypes.byref(q), ctypes.byref(ms)), "scc_batch_autotune")
        return t.value, q.value, ms.value

    def run(self, algo="h", t1=True, t2=True, warp=1, labels=True, sequential=False, out=None, check=True):
        """Returns (labels concatenated in batch order or None, per-graph results, stats)."""
        flags = (N.FLAG_TRIM1 if t1 else 0) | (N.FLAG_TRIM2 if t2 else 0)
        flags |= N.FLAG_BATCH_SEQUENTIAL if sequential else 0
        if labels and out is None:
            out = np.zeros(max(self.total_vertices, 1), dtype=np.uint32)
        res = (N.BatchResult * max(len(self.graphs), 1))()
        st = N.Stats()
        rc = self._lib.scc_batch_run(self._h, _algo_code(algo), flags, int(warp), _ptr(out) if labels else None,
                                     res, ctypes.byref(st))
        if check:
            N.check(rc, "scc_batch_run")
        results = [(int(r.num_sccs), int(r.num_trim1), int(r.status)) for r in res[:len(self.graphs)]]
        return (out[:self.total_vertices] if labels else None), results, st.as_dict()

    def labels_of(self, labels, i):
        return labels[self.offsets[i]:self.offsets[i + 1]]


class Server:
    """Request server: continuous batching under a device-memory budget.

    submit() queues one host graph and the host array its labels go to;
    both must stay alive until the request's result has been polled.
    """

    def __init__(self, device: int = 0, algo="h", t1=True, t2=True, warp=1, budget_bytes: int = 0, lanes: int = 0,
                 max_graphs_per_batch: int = 0, large_vertices: int = 0, batch_threads: int = 0, qcap: int = 0,
                 cluster: int = 0, big_vertices: int = 0, large_cluster: int = 0):
        self._lib = N.lib()
        cfg = N.ServerConfig(int(budget_bytes), int(lanes), int(max_graphs_per_batch), int(large_vertices),
                             int(batch_threads), int(qcap), _algo_code(algo),
                             (N.FLAG_TRIM1 if t1 else 0) | (N.FLAG_TRIM2 if t2 else 0), int(warp),
                             int(cluster), int(big_vertices), int(large_cluster))
        h = ctypes.c_void_p()
        N.check(self._lib.scc_server_create(int(device), ctypes.byref(cfg), ctypes.byref(h)), "scc_server_create")
        self._h = h
        self._live = {}   # ticket -> (graph, labels) kept alive until polled

    def submit(self, g: Graph, out: Optional[np.ndarray] = None) -> int:
        if out is None:
            out = np.zeros(max(g.V, 1), dtype=np.uint32)
        view = N.CsrView(g.V, g.E, _ptr(g.Fr), _ptr(g.Fc), _ptr(g.Br), _ptr(g.Bc))
        t = ctypes.c_uint64(0)
        N.check(self._lib.scc_server_submit(self._h, ctypes.byref(view), _ptr(out), ctypes.byref(t)), "scc_server_submit")
        self._live[t.value] = (g, out)
        return t.value

    def poll(self, max_results: int = 1024, wait_ms: int = 0):
        """Finished requests: list of dicts with ticket, status, counts, latency and the labels array."""
        buf = (N.ServerResult * max_results)()
        n = ctypes.c_uint32(0)
        N.check(self._lib.scc_server_poll(self._h, buf, max_results, ctypes.byref(n), int(wait_ms)))
        out = []
        for r in buf[:n.value]:
            g, lab = self._live.pop(r.ticket, (None, None))
            out.append({"ticket": r.ticket, "status": r.status, "num_sccs": r.num_sccs, "num_trim1": r.num_trim1,
                        "latency_ms": r.latency_ms, "queue_ms": r.queue_ms, "lane": r.lane,
                        "labels": lab[:g.V] if g is not None else None})
        return out

    def info(self):
        a, b, c, d = (ctypes.c_uint64(0) for _ in range(4))
        N.check(self._lib.scc_server_info(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d)))
        return {"pending": a.value, "completed": b.value, "held_bytes": c.value, "rejected": d.value}

    def launches(self) -> int:
        """Kernel launches made so far."""
        n = ctypes.c_uint64(0)
        N.check(self._lib.scc_server_launches(self._h, ctypes.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.scc_server_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------------
# graph files
# ----------------------------------------------------------------------
def _take_host_graph(hg: N.HostGraph, name: str = "") -> Graph:
    V, E = int(hg.V), int(hg.E)
    Fr = np.ctypeslib.as_array(hg.Fr, shape=(V + 2,)).copy()
    Br = np.ctypeslib.as_array(hg.Br, shape=(V + 2,)).copy()
    Fc = np.ctypeslib.as_array(hg.Fc, shape=(max(E, 1),))[:E].copy()
    Bc = np.ctypeslib.as_array(hg.Bc, shape=(max(E, 1),))[:E].copy()
    N.lib().scc_free_host_graph(ctypes.byref(hg))
    return Graph(V, E, Fr, Fc, Br, Bc, name)


def load_graph(path: str) -> Graph:
    """GTgraph text (the reference's format) or the binary CSR format."""
    hg = N.HostGraph()
    N.check(N.lib().scc_load_graph(path.encode(), ctypes.byref(hg)), f"load {path}")
    return _take_host_graph(hg, path)


def graph_from_arcs(V: int, src, dst, name: str = "") -> Graph:
    """Forward + reverse CSR from 1-based arcs, ordered as the reference loader orders them."""
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    hg = N.HostGraph()
    N.check(N.lib().scc_graph_from_arcs(int(V), int(src.shape[0]), _ptr(src), _ptr(dst), ctypes.byref(hg)),
            "scc_graph_from_arcs")
    return _take_host_graph(hg, name)


def save_binary(path: str, g: Graph) -> None:
    hg = N.HostGraph(g.V, g.E, g.Fr.ctypes.data_as(N.u32p), g.Fc.ctypes.data_as(N.u32p),
                     g.Br.ctypes.data_as(N.u32p), g.Bc.ctypes.data_as(N.u32p), None)
    N.check(N.lib().scc_save_binary(path.encode(), ctypes.byref(hg)), f"save {path}")


def save_gtgraph(path: str, g: Graph) -> None:
    """Write g as GTgraph text (the reference's input format, load.cpp:12-45)."""
    hg = N.HostGraph(g.V, g.E, g.Fr.ctypes.data_as(N.u32p), g.Fc.ctypes.data_as(N.u32p),
                     g.Br.ctypes.data_as(N.u32p), g.Bc.ctypes.data_as(N.u32p), None)
    N.check(N.lib().scc_save_gtgraph(path.encode(), ctypes.byref(hg)), f"save {path}")


def save_metis(path: str, g: Graph) -> None:
    """Write g in the reference converter's METIS input layout (MetisInput.cpp:114-131)."""
    hg = N.HostGraph(g.V, g.E, g.Fr.ctypes.data_as(N.u32p), g.Fc.ctypes.data_as(N.u32p),
                     g.Br.ctypes.data_as(N.u32p), g.Bc.ctypes.data_as(N.u32p), None)
    N.check(N.lib().scc_save_metis(path.encode(), ctypes.byref(hg)), f"save {path}")


def load_partition(path: str, V: int) -> np.ndarray:
    """METIS partition ids as Pr[0..V+1] (Pr[v] for vertex v; load.cpp:115-130)."""
    Pr = np.zeros(V + 2, dtype=np.uint32)
    N.check(N.lib().scc_load_partition(path.encode(), int(V), _ptr(Pr)), f"load {path}")
    return Pr


def loadFullGraph(filename: str):
    """The reference's loader: returns (CSize, RSize, Fc, Fr, Bc, Br, Pr).

    Pr (METIS partition ids, read only by the reference's detectSCC) comes
    from the file named by SCC_METIS_PARTITION when it is set (the
    reference reads a fixed path, load.cpp:115-130), else it is zero-filled.
    """
    import os
    g = load_graph(filename)
    part = os.environ.get("SCC_METIS_PARTITION")
    Pr = load_partition(part, g.V) if part else np.zeros(g.V + 2, dtype=np.uint32)
    return g.E, g.V, g.Fc, g.Fr, g.Bc, g.Br, Pr


# ----------------------------------------------------------------------
# reference drivers (print like the reference, return the count)
# ----------------------------------------------------------------------
def _reference_call(algo: str, CSize, RSize, Fc, Fr, Bc, Br, t1, t2, warpSize=1) -> int:
    arrs = [np.ascontiguousarray(a, dtype=np.uint32) for a in (Fc, Fr, Bc, Br)]
    n = ctypes.c_uint64(0)
    rc = N.lib().scc_reference_call(ord(algo), int(CSize), int(RSize), _ptr(arrs[0]), _ptr(arrs[1]),
                                    _ptr(arrs[2]), _ptr(arrs[3]), int(bool(t1)), int(bool(t2)),
                                    int(warpSize), ctypes.byref(n))
    if rc == 3:  # out of device memory: the reference throws this message
        raise MemoryError("Error: Not enough memory on GPU\n")
    N.check(rc, ALGOS[algo])
    return int(n.value)


def vHong(CSize, RSize, Fc, Fr, Bc, Br, t1=True, t2=True) -> int:
    return _reference_call("g", CSize, RSize, Fc, Fr, Bc, Br, t1, t2)


def vSlota(CSize, RSize, Fc, Fr, Bc, Br, t1=True, t2=True) -> int:
    return _reference_call("h", CSize, RSize, Fc, Fr, Bc, Br, t1, t2)


def wHong(CSize, RSize, Fc, Fr, Bc, Br, t1=True, t2=True, warpSize=1) -> int:
    return _reference_call("x", CSize, RSize, Fc, Fr, Bc, Br, t1, t2, warpSize)


def wSlota(CSize, RSize, Fc, Fr, Bc, Br, t1=True, t2=True, warpSize=1) -> int:
    return _reference_call("y", CSize, RSize, Fc, Fr, Bc, Br, t1, t2, warpSize)
