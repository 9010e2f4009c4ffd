"""Record the reference binary's own outputs on the golden fixtures.

Run on a machine with a B200 after `make -C oracle ref` built
oracle/_ref/scc_ref (the reference's unchanged scc.cu / scc_kernels.cu /
scc_WCC.cu / scc_Coloring.cu linked with a project-written loader):

    python tests/golden/make_ref_counts.py [output.json]

For every fixture and every driver configuration it runs the reference CLI,
parses "Number Of Sccs", "numberOf1Sccs" (vHong only) and "Time", and
writes tests/golden/ref_counts.json.  vHong / wHong with -p 0 are not run:
a range made only of vertices with in-degree x out-degree = 0 never gets a
pivot there and the reference's host loop does not end.
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = os.path.join(ROOT, "oracle", "_ref", "scc_ref")
FIXTURES = ["sample0", "sample4", "sample5", "sample1", "sample128", "sample2"]
CONFIGS = [("g", 1, 0, 1), ("g", 1, 1, 1), ("x", 1, 0, 8), ("x", 1, 1, 32),
           ("h", 1, 1, 1), ("h", 0, 0, 1), ("y", 1, 1, 8), ("y", 0, 1, 4)]


def run_reference(path: str, algo: str, p: int, q: int, w: int, timeout: float = 120.0):
    out = subprocess.run([REF, "-a", algo, "-p", str(p), "-q", str(q), "-w", str(w), "-f", path],
                         capture_output=True, text=True, timeout=timeout)
    text = out.stdout
    m = re.search(r"Number Of Sccs : (-?\d+)", text)
    t = re.search(r"Time : ([0-9.]+)", text)
    o = re.search(r"numberOf1Sccs: (-?\d+)", text)
    return {"rc": out.returncode, "num_sccs": int(m.group(1)) if m else None,
            "numberOf1Sccs": int(o.group(1)) if o else None, "time_ms": float(t.group(1)) if t else None,
            "stdout": text}


def main():
    from oracle.gtgraph_ref import write_gtgraph
    res = {}
    with tempfile.TemporaryDirectory() as td:
        for name in FIXTURES:
            z = np.load(os.path.join(HERE, name + ".npz"))
            path = os.path.join(td, name + ".gr")
            write_gtgraph(path, int(z["V"]), z["src"], z["dst"], name)
            for algo, p, q, w in CONFIGS:
                r = run_reference(path, algo, p, q, w)
                key = f"{name}:{algo}:p{p}:q{q}:w{w}"
                r.pop("stdout")
                res[key] = r
                print(key, r, flush=True)
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_counts.json")
    with open(out, "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
