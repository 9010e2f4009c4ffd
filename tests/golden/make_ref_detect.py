"""Record the reference binary's own detectSCC (-a d) outputs.

Run on a machine with a B200 after `make -C oracle ref`:

    python tests/golden/make_ref_detect.py [output.json]

detectSCC (scc_WCC.cu:1000-1617) partitions the graph with the METIS
partition file its loader reads (load.cpp:115-130; the harness loader takes
the path from SCC_METIS_PARTITION).  For every shipped sample that has a
shipped partition file with ids below the driver's fixed partition count of
10 (scc_WCC.cu:1035; larger ids would index past its pivot tables), and with
no partition file at all (every vertex in partition 0), it runs
`scc_ref -a d -p 1 -q Q -w 1` three times and records stdout with the time
value masked, so that a run-to-run difference shows.  -p 0 is not run: a
range of vertices with in-degree x out-degree = 0 never gets a pivot there
and the driver's host loop does not end.  Writes
tests/golden/ref_detect.json.
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
CASES = [("sample0", "sample0.part.2"), ("sample4", "sample4.part.3"), ("sample5", "sample5.part.5"),
         ("sample1", "sample1.part.10"), ("sample128", "sample128.part.10"),
         ("sample0", None), ("sample4", None), ("sample5", None), ("sample1", None), ("sample128", None)]


def main():
    from oracle.gtgraph_ref import write_gtgraph
    parts = np.load(os.path.join(HERE, "metis_partitions.npz"))
    res = {}
    with tempfile.TemporaryDirectory() as td:
        for name, part in CASES:
            z = np.load(os.path.join(HERE, name + ".npz"))
            path = os.path.join(td, name + ".gr")
            write_gtgraph(path, int(z["V"]), z["src"], z["dst"], name)
            env = dict(os.environ)
            env.pop("SCC_METIS_PARTITION", None)
            if part:
                ids = parts[part]
                if int(ids.max()) >= 10:
                    continue
                pp = os.path.join(td, part)
                with open(pp, "w") as f:
                    f.write("\n".join(str(int(x)) for x in ids) + "\n")
                env["SCC_METIS_PARTITION"] = pp
            for q in (0, 1):
                outs = []
                for _ in range(3):
                    r = subprocess.run([REF, "-a", "d", "-p", "1", "-q", str(q), "-w", "1", "-f", path],
                                       capture_output=True, text=True, timeout=120, env=env)
                    outs.append({"rc": r.returncode, "stdout": re.sub(r"Time : [0-9.]+", "Time : T", r.stdout)})
                key = f"{name}:{part or 'none'}:q{q}"
                m = re.search(r"Number Of Sccs : (-?\d+)", outs[0]["stdout"])
                res[key] = {"num_sccs": int(m.group(1)) if m else None, "runs": outs,
                            "stable": all(o == outs[0] for o in outs)}
                print(key, res[key]["num_sccs"], res[key]["stable"], flush=True)
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_detect.json")
    with open(out, "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
