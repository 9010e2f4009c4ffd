"""Generate the golden SCC fixtures from the reference's sample graphs.

Run once in a container that has the reference checkout (it is read, never
modified):

    python tests/golden/make_golden.py /root/reference/data

For every GTgraph sample in the reference's ``data/`` folder (the ``*.gr~``
editor backups are skipped) this script

1. parses the file exactly as the reference loader does
   (``oracle/gtgraph_ref.py``, restating ``src/load.cpp:12-113``);
2. computes the strongly connected components twice, independently of the
   project's own code: with ``scipy.sparse.csgraph.connected_components``
   (connection='strong') and with ``networkx.strongly_connected_components``;
3. checks the two agree, canonicalises the labels to the minimum vertex id
   of each component, and writes ``tests/golden/<name>.npz`` holding the edge
   list as read (file order), V, E, the canonical labels and the counts.

The fixtures are what the CPU tests pin the oracle against; the GPU tests
pin the CUDA engine against the same files.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle.gtgraph_ref import parse_gtgraph_text  # noqa: E402

SAMPLES = ["sample0.gr", "sample4.gr", "sample5.gr", "sample1.gr", "sample128.gr", "sample2.gr"]


def canonical(labels_1based: np.ndarray) -> np.ndarray:
    """Map arbitrary component ids (index v-1 -> comp) to min-vertex-id labels."""
    V = labels_1based.shape[0]
    mn = np.full(labels_1based.max() + 1 if V else 1, np.iinfo(np.int64).max, dtype=np.int64)
    ids = np.arange(1, V + 1, dtype=np.int64)
    np.minimum.at(mn, labels_1based, ids)
    return mn[labels_1based]


def scc_scipy(V, src, dst):
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    A = sp.coo_matrix((np.ones(len(src)), (src - 1, dst - 1)), shape=(V, V)).tocsr()
    n, lab = connected_components(A, directed=True, connection="strong")
    return n, canonical(lab.astype(np.int64))


def scc_networkx(V, src, dst):
    import networkx as nx
    G = nx.DiGraph()
    G.add_nodes_from(range(1, V + 1))
    G.add_edges_from(zip(src.tolist(), dst.tolist()))
    lab = np.zeros(V, dtype=np.int64)
    n = 0
    for comp in nx.strongly_connected_components(G):
        m = min(comp)
        for v in comp:
            lab[v - 1] = m
        n += 1
    return n, lab


def main(data_dir: str) -> None:
    summary = {}
    for name in SAMPLES:
        path = os.path.join(data_dir, name)
        with open(path) as f:
            V, E, src, dst = parse_gtgraph_text(f.read())
        n1, lab1 = scc_scipy(V, src, dst)
        n2, lab2 = scc_networkx(V, src, dst)
        assert n1 == n2 and np.array_equal(lab1, lab2), name
        sizes = np.bincount(lab1, minlength=V + 1)
        sizes = sizes[sizes > 0]
        pairs = np.stack([src, dst], 1)
        dups = int(len(pairs) - len(np.unique(pairs, axis=0))) if E else 0
        out = os.path.join(HERE, name.replace(".gr", ".npz"))
        np.savez_compressed(out, V=np.int64(V), E=np.int64(E),
                            src=src.astype(np.uint32), dst=dst.astype(np.uint32),
                            labels=lab1.astype(np.uint32), nscc=np.int64(n1))
        summary[name] = {"V": V, "E": E, "dups": dups, "nscc": int(n1),
                         "size1": int((sizes == 1).sum()), "size2": int((sizes == 2).sum()),
                         "largest": int(sizes.max()) if len(sizes) else 0}
        print(name, summary[name])
    with open(os.path.join(HERE, "golden_summary.json"), "w") as f:
        json.dump(summary, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.environ.get("SCC_REFERENCE_DIR", "/root/reference"), "data"))
