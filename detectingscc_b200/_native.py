"""ctypes binding of libscc_b200.so (include/scc_b200.h).

The library is built in-tree (``python -m detectingscc_b200.build``).  There
is no fallback: if the library is missing or cannot be loaded every entry
point raises ``NativeLibraryError``.
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libscc_b200.so")
CLI_PATH = os.path.join(_PKG, "bin", "scc")
METIS_CLI_PATH = os.path.join(_PKG, "bin", "scc_metis")

u32 = ctypes.c_uint32
u64 = ctypes.c_uint64
u32p = ctypes.POINTER(ctypes.c_uint32)


class NativeLibraryError(RuntimeError):
    pass


class CsrView(ctypes.Structure):
    _fields_ = [("num_vertices", u32), ("num_edges", u32),
                ("Fr", ctypes.c_void_p), ("Fc", ctypes.c_void_p),
                ("Br", ctypes.c_void_p), ("Bc", ctypes.c_void_p)]


class Stats(ctypes.Structure):
    _fields_ = [("num_sccs", u64), ("num_trim1", u64), ("num_trim2", u64), ("num_pivot", u64),
                ("edges_scanned", u64), ("vertex_visits", u64),
                ("passes", u32), ("outer_iters", u32), ("tail_pass", u32), ("gpu_launches", u32),
                ("grid_blocks", u32), ("used_block_path", u32),
                ("kernel_ms", ctypes.c_float), ("total_ms", ctypes.c_float),
                ("error_where", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class HostGraph(ctypes.Structure):
    _fields_ = [("V", u32), ("E", u32), ("Fr", u32p), ("Fc", u32p), ("Br", u32p), ("Bc", u32p),
                ("Pr", u32p)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("budget_bytes", u64), ("lanes", u32), ("max_graphs_per_batch", u32), ("large_vertices", u32),
                ("batch_threads", ctypes.c_int32), ("qcap", u32), ("algo", ctypes.c_int32), ("flags", u32),
                ("warp_width", ctypes.c_int32), ("cluster", u32), ("big_vertices", u32), ("large_cluster", u32)]


class ServerResult(ctypes.Structure):
    _fields_ = [("ticket", u64), ("status", ctypes.c_int32), ("num_vertices", u32), ("num_sccs", u64),
                ("num_trim1", u64), ("latency_ms", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("lane", ctypes.c_int32), ("reserved", u32)]


class DetectResult(ctypes.Structure):
    _fields_ = [("num_sccs", u64), ("num_trim1", u64), ("num_trim2", u64), ("num_ranges", u64),
                ("merge_rounds", u32), ("nospace_mask", u32)]


class BatchResult(ctypes.Structure):
    _fields_ = [("num_sccs", u64), ("num_trim1", u64), ("status", ctypes.c_int32), ("reserved", u32)]


# status codes (scc_status)
SCC_OK = 0
STATUS_NAMES = {0: "SCC_OK", 1: "SCC_ERR_INVALID_ARG", 2: "SCC_ERR_CUDA", 3: "SCC_ERR_OOM",
                4: "SCC_ERR_TOO_LARGE", 5: "SCC_ERR_NO_DEVICE", 6: "SCC_ERR_BUDGET", 7: "SCC_ERR_IO",
                20: "SCC_ERR_OVERFLOW", 21: "SCC_ERR_NOT_CONVERGED", 22: "SCC_ERR_TIMEOUT",
                23: "SCC_ERR_BAD_GRAPH"}

FLAG_TRIM1 = 0x1
FLAG_TRIM2 = 0x2
FLAG_DEVICE = 0x4
FLAG_INSTRUMENT = 0x8
FLAG_FORCE_GRID = 0x10
FLAG_FORCE_BLOCK = 0x20
FLAG_DERIVE_REVERSE = 0x80
FLAG_BATCH_SEQUENTIAL = 0x40
MAX_VERTICES = 268435454

# every symbol include/scc_b200.h and include/scc_compat.h declare
C_SYMBOLS = ["scc_create", "scc_destroy", "scc_run", "scc_set_tuning", "scc_status_string",
             "scc_version", "scc_get_trace", "scc_derive_reverse", "scc_load_graph", "scc_save_binary", "scc_graph_from_arcs",
             "scc_free_host_graph", "scc_run_async", "scc_finish", "scc_save_gtgraph", "scc_load_graph_device", "scc_save_metis", "scc_load_partition", "scc_detect", "scc_reference_detect",
             "scc_reference_call", "scc_batch_create", "scc_batch_run",
             "scc_batch_destroy", "scc_run_noalloc", "scc_batch_set_schedule", "scc_batch_get_schedule",
             "scc_batch_autotune", "scc_batch_info", "scc_batch_set_cluster", "scc_batch_get_cluster", "scc_server_create", "scc_server_submit",
             "scc_server_poll", "scc_server_info", "scc_server_launches", "scc_server_destroy"]
CXX_SYMBOLS = ["_Z5vHongjjPjS_S_S_bb", "_Z6vSlotajjPjS_S_S_bb", "_Z5wHongjjPjS_S_S_bbi",
               "_Z6wSlotajjPjS_S_S_bbi", "_Z13loadFullGraphPKcPjS1_PS1_S2_S2_S2_S2_", "_Z9detectSCCjjPjS_S_S_S_bb"]

_lib = None


class SCCError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        name = STATUS_NAMES.get(code, str(code))
        msg = f"{name}: {status_string(code)}" if _lib is not None else name
        super().__init__(f"{what}: {msg}" if what else msg)


def lib():
    """Load the native library (raises NativeLibraryError if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NativeLibraryError(
            f"{LIB_PATH} is missing; build it with `python -m detectingscc_b200.build`")
    try:
        L = ctypes.CDLL(LIB_PATH)
    except OSError as e:  # pragma: no cover - environment specific
        raise NativeLibraryError(f"cannot load {LIB_PATH}: {e}") from e
    vp = ctypes.c_void_p
    L.scc_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    L.scc_destroy.argtypes = [vp]
    L.scc_run.argtypes = [vp, ctypes.POINTER(CsrView), ctypes.c_int, u32, ctypes.c_int, vp,
                          ctypes.POINTER(Stats), vp]
    L.scc_run_async.argtypes = [vp, ctypes.POINTER(CsrView), ctypes.c_int, u32, ctypes.c_int, vp, vp]
    L.scc_finish.argtypes = [vp, ctypes.POINTER(Stats)]
    L.scc_set_tuning.argtypes = [vp, ctypes.c_char_p, ctypes.c_longlong]
    L.scc_status_string.restype = ctypes.c_char_p
    L.scc_status_string.argtypes = [ctypes.c_int]
    L.scc_version.restype = ctypes.c_char_p
    L.scc_load_graph.argtypes = [ctypes.c_char_p, ctypes.POINTER(HostGraph)]
    L.scc_save_binary.argtypes = [ctypes.c_char_p, ctypes.POINTER(HostGraph)]
    L.scc_graph_from_arcs.argtypes = [u32, u64, vp, vp, ctypes.POINTER(HostGraph)]
    L.scc_save_metis.argtypes = [ctypes.c_char_p, ctypes.POINTER(HostGraph)]
    L.scc_save_gtgraph.argtypes = [ctypes.c_char_p, ctypes.POINTER(HostGraph)]
    L.scc_load_graph_device.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(CsrView), vp]
    L.scc_detect.argtypes = [vp, ctypes.POINTER(CsrView), vp, u32, ctypes.POINTER(DetectResult)]
    L.scc_reference_detect.argtypes = [u32, u32, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(u64)]
    L.scc_load_partition.argtypes = [ctypes.c_char_p, u32, vp]
    L.scc_free_host_graph.argtypes = [ctypes.POINTER(HostGraph)]
    L.scc_free_host_graph.restype = None
    L.scc_reference_call.argtypes = [ctypes.c_int, u32, u32, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.POINTER(u64)]
    L.scc_batch_create.argtypes = [vp, ctypes.POINTER(CsrView), u32, ctypes.POINTER(vp)]
    L.scc_batch_run.argtypes = [vp, ctypes.c_int, u32, ctypes.c_int, vp, ctypes.POINTER(BatchResult),
                                ctypes.POINTER(Stats)]
    L.scc_batch_destroy.argtypes = [vp]
    L.scc_batch_set_schedule.argtypes = [vp, ctypes.c_int, u32]
    L.scc_batch_get_schedule.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(u32)]
    L.scc_batch_autotune.argtypes = [vp, ctypes.c_int, u32, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(u32), ctypes.POINTER(ctypes.c_float)]
    L.scc_batch_info.argtypes = [vp, ctypes.POINTER(u64), ctypes.POINTER(u64), ctypes.POINTER(u32)]
    L.scc_batch_set_cluster.argtypes = [vp, ctypes.c_int, u32]
    L.scc_batch_get_cluster.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(u32), ctypes.POINTER(u32)]
    L.scc_run_noalloc.argtypes = [ctypes.POINTER(CsrView), ctypes.c_int, u32, ctypes.c_int, vp,
                                  ctypes.POINTER(Stats), vp]
    L.scc_server_create.argtypes = [ctypes.c_int, ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
    L.scc_server_submit.argtypes = [vp, ctypes.POINTER(CsrView), vp, ctypes.POINTER(u64)]
    L.scc_server_poll.argtypes = [vp, ctypes.POINTER(ServerResult), u32, ctypes.POINTER(u32), ctypes.c_int]
    L.scc_server_info.argtypes = [vp, ctypes.POINTER(u64), ctypes.POINTER(u64), ctypes.POINTER(u64), ctypes.POINTER(u64)]
    L.scc_server_launches.argtypes = [vp, ctypes.POINTER(u64)]
    L.scc_server_destroy.argtypes = [vp]
    L.scc_derive_reverse.argtypes = [vp, vp, vp, u32, u32, vp, vp, vp]
    L.scc_get_trace.argtypes = [vp, ctypes.POINTER(u64), u32, ctypes.POINTER(u32), ctypes.POINTER(u64)]
    _lib = L
    return L


def status_string(code: int) -> str:
    return lib().scc_status_string(int(code)).decode()


def check(code: int, what: str = "") -> None:
    if code != SCC_OK:
        raise SCCError(code, what)
