"""Build the native library and the CLI in-tree (no GPU needed).

    python -m detectingscc_b200.build [--force]

Produces
    detectingscc_b200/libscc_b200.so   C ABI (include/scc_b200.h) and the
                                       reference-signature shims
                                       (include/scc_compat.h)
    detectingscc_b200/bin/scc          the drop-in command line
    detectingscc_b200/bin/scc_metis    the METIS input converter (MetisInput.cpp)

CUDA code is compiled for sm_100a only; the CUDA runtime is linked
statically so the library does not depend on which libcudart a host
process (e.g. PyTorch) has loaded.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libscc_b200.so")
CLI = os.path.join(PKG, "bin", "scc")
CLI_METIS = os.path.join(PKG, "bin", "scc_metis")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-I/usr/local/cuda/include"]

CU_SOURCES = ["scc_engine.cu", "scc_batch.cu", "scc_noalloc.cu", "scc_serve.cu", "scc_transpose.cu", "scc_detect.cu"]
CXX_LIB_SOURCES = ["gtgraph_load.cpp", "scc_compat.cpp"]
CXX_CLI_SOURCES = ["scc_cli.cpp", "scc_metis_cli.cpp"]
HEADERS = ["scc_device.cuh", "scc_phases.cuh", "scc_internal.h", "scc_host.h", "scc_batch_internal.h"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "scc_b200.h"), os.path.join(ROOT, "include", "scc_compat.h")]
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(BUILD, src + ".o")
        if force or _newer(o, [s] + hdrs):
            extra = ["-Xptxas", "-v"] if verbose_ptxas else []
            jobs.append([NVCC] + CU_FLAGS + extra + ["-c", s, "-o", o])
        objs.append(o)
    # the translation units are independent: compile them concurrently
    with cf.ThreadPoolExecutor(max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, j) for j in jobs]:
            f.result()
    lib_objs = []
    for src in CXX_LIB_SOURCES + CXX_CLI_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _newer(o, [s] + hdrs):
            _run(["g++"] + CXX_FLAGS + ["-c", s, "-o", o])
        if src in CXX_LIB_SOURCES:
            lib_objs.append(o)
    all_lib = objs + lib_objs
    if force or _newer(LIB, all_lib):
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + all_lib + ["-lpthread"])
    for exe, src in ((CLI, "scc_cli.cpp"), (CLI_METIS, "scc_metis_cli.cpp")):
        cli_obj = os.path.join(BUILD, src + ".o")
        if force or _newer(exe, all_lib + [cli_obj]):
            _run([NVCC] + ARCH + ["-o", exe, cli_obj] + all_lib + ["-lpthread"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
