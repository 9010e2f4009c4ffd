"""B200-native SCC engine: a drop-in for Amit104/DetectingSCC's vHong /
vSlota / wHong / wSlota drivers, its GTgraph loader and its ./scc CLI.

The compute path is the native library ``libscc_b200.so`` (hand-written
sm_100a CUDA behind a C ABI, ``include/scc_b200.h``); this package is its
Python host mirror.  There is no CPU fallback: without the library every
call raises ``NativeLibraryError``.
"""
from ._native import NativeLibraryError, SCCError  # noqa: F401
from .api import (ALGOS, Batch, Engine, Graph, Result, Server, graph_from_arcs, load_graph,  # noqa: F401
                  load_partition, loadFullGraph, save_binary, save_gtgraph, save_metis, vHong, vSlota, wHong,
                  wSlota)

__all__ = ["Batch", "Engine", "Server", "Graph", "Result", "graph_from_arcs", "load_graph", "loadFullGraph",
           "save_binary", "save_gtgraph", "save_metis", "load_partition", "vHong", "vSlota", "wHong", "wSlota", "NativeLibraryError", "SCCError",
           "ALGOS"]
