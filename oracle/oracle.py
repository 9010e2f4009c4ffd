"""ctypes front end of the C oracle (``oracle/scc_oracle.c``).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by the smoke check and by
bench.py's CPU-baseline leg; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with gcc -O3 (no GPU needed)."""
    src = os.path.join(_HERE, "scc_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O3", "-march=x86-64-v2", "-fPIC", "-shared",
                               "-o", _LIB_PATH, src])
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        lib.oracle_tarjan.restype = ctypes.c_longlong
        lib.oracle_tarjan.argtypes = [ctypes.c_uint32, u32p, u32p, u32p]
        for fn in (lib.oracle_hong, lib.oracle_slota):
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_uint32, u32p, u32p, u32p, u32p,
                           ctypes.c_int, ctypes.c_int, u32p, u64p]
        lib.oracle_detect.restype = ctypes.c_int
        lib.oracle_detect.argtypes = [ctypes.c_uint32, u32p, u32p, u32p, u32p, u32p, ctypes.c_int, ctypes.c_int,
                                      u64p, u32p, u32p]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def tarjan(V, Fr, Fc):
    """Canonical labels (V+1 entries, [0] = 0) and the SCC count."""
    lib = _load()
    Fr = np.ascontiguousarray(Fr, dtype=np.uint32)
    Fc = np.ascontiguousarray(Fc, dtype=np.uint32)
    if Fc.size == 0:
        Fc = np.zeros(1, np.uint32)
    labels = np.zeros(V + 1, dtype=np.uint32)
    n = lib.oracle_tarjan(V, _p(Fr), _p(Fc), _p(labels))
    if n < 0:
        raise MemoryError("oracle_tarjan out of memory")
    return labels, int(n)


def time_tarjan(V, Fr, Fc, budget_s: float = 20.0, max_reps: int = 5):
    """Time repeated Tarjan runs on one host core; returns (seconds/run, reps)."""
    lib = _load()
    Fr = np.ascontiguousarray(Fr, dtype=np.uint32)
    Fc = np.ascontiguousarray(Fc, dtype=np.uint32)
    labels = np.zeros(V + 1, dtype=np.uint32)
    times = []
    t_start = time.perf_counter()
    while len(times) < max_reps:
        t0 = time.perf_counter()
        lib.oracle_tarjan(V, _p(Fr), _p(Fc), _p(labels))
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s:
            break
    return float(np.median(times)), len(times)


def _phase(fn, V, Fr, Fc, Br, Bc, t1, t2):
    Fr = np.ascontiguousarray(Fr, dtype=np.uint32)
    Fc = np.ascontiguousarray(Fc, dtype=np.uint32)
    Br = np.ascontiguousarray(Br, dtype=np.uint32)
    Bc = np.ascontiguousarray(Bc, dtype=np.uint32)
    if Fc.size == 0:
        Fc = np.zeros(1, np.uint32)
        Bc = np.zeros(1, np.uint32)
    labels = np.zeros(V + 1, dtype=np.uint32)
    counts = np.zeros(3, dtype=np.uint64)
    rc = fn(V, _p(Fr), _p(Fc), _p(Br), _p(Bc), int(bool(t1)), int(bool(t2)), _p(labels),
            counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    if rc != 0:
        raise MemoryError("oracle out of memory")
    return labels, [int(c) for c in counts]


def hong(V, Fr, Fc, Br, Bc, t1=True, t2=True):
    """Restated vHong/wHong: (labels, [trim1, trim2_pairs, pivots])."""
    return _phase(_load().oracle_hong, V, Fr, Fc, Br, Bc, t1, t2)


def slota(V, Fr, Fc, Br, Bc, t1=True, t2=True):
    """Restated vSlota/wSlota: (labels, [trim1, 0, pivots])."""
    return _phase(_load().oracle_slota, V, Fr, Fc, Br, Bc, t1, t2)


DETECT_HEAD = ("LOCAL SCC's IDENTIFIED! NODES WITH SAME RANGE VALUES BELONG TO THE SAME SCC!!\n"
               "Fs AND Bs ARE POPULATED!!\nSTARTING MERGE!\n")


def detect(V, Fr, Fc, Br, Bc, Pr, t1=True, t2=True):
    """Restated detectSCC (-a d): ([trim1, trim2, distinct ranges], merge rounds, "No space!" round mask)."""
    lib = _load()
    arrs = [np.ascontiguousarray(a, dtype=np.uint32) for a in (Fr, Fc, Br, Bc)]
    arrs = [a if a.size else np.zeros(1, np.uint32) for a in arrs]
    Pr = np.ascontiguousarray(Pr, dtype=np.uint32)
    if Pr.size < V + 2:
        Pr = np.concatenate([Pr, np.zeros(V + 2 - Pr.size, np.uint32)])
    counts = np.zeros(3, dtype=np.uint64)
    rounds = ctypes.c_uint32(0)
    nospace = ctypes.c_uint32(0)
    rc = lib.oracle_detect(V, *(_p(a) for a in arrs), _p(Pr), int(bool(t1)), int(bool(t2)),
                           counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), ctypes.byref(rounds),
                           ctypes.byref(nospace))
    if rc == 3:
        raise MemoryError("oracle out of memory")
    if rc != 0:
        raise RuntimeError("detectSCC restatement: local loop did not converge")
    return [int(c) for c in counts], int(rounds.value), int(nospace.value)


def detect_stdout(counts, rounds, nospace, time_text="T"):
    """The text the reference's detectSCC prints, then main's newline (scc_WCC.cu:1264-1561, scc.cu:109)."""
    out = DETECT_HEAD
    for r in range(1, rounds + 1):
        out += f"Iterations {r}\n"
        if r <= 32 and (nospace >> (r - 1)) & 1:
            out += "No space!\n"
    out += "MERGING DONE! ^_^\n"
    out += f"\nNumber Of Sccs : {sum(counts)}\nTime : {time_text}\n\n"
    return out
