"""Golden vectors for the METIS input converter and the METIS partitions.

    python tests/golden/make_metis_golden.py [REFERENCE_DIR]

The reference ships, beside its sample graphs data/sampleN.gr, the files its
converter tool wrote from them (src/MeTiSInputN.graph, MetisInput.cpp) and
METIS partitions of those (src/MeTiSInputN.graph.part.K).  This script
records, per sample, the SHA-256 and size of the converter output (with the
CRLF line ends some of the shipped copies carry turned back into the "\\n"
the tool writes) into tests/golden/metis_golden.json, and the partition ids
into tests/golden/metis_partitions.npz.
Test infrastructure only; run where the reference checkout exists.
"""
import glob
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref: str) -> None:
    out = {"converter": {}, "partitions": {}}
    ids = {}
    for path in sorted(glob.glob(os.path.join(ref, "src", "MeTiSInput*.graph"))):
        n = os.path.basename(path)[len("MeTiSInput"):-len(".graph")]
        sample = os.path.join(ref, "data", f"sample{n}.gr")
        if not os.path.exists(sample):
            continue   # written from a graph the reference does not ship
        data = open(path, "rb").read().replace(b"\r\n", b"\n")
        out["converter"][f"sample{n}"] = {"sha256": hashlib.sha256(data).hexdigest(), "bytes": len(data),
                                          "source": f"src/MeTiSInput{n}.graph"}
    for path in sorted(glob.glob(os.path.join(ref, "src", "MeTiSInput*.graph.part.*"))):
        base = os.path.basename(path)
        n = base[len("MeTiSInput"):base.index(".graph")]
        k = int(base.rsplit(".", 1)[1])
        if not os.path.exists(os.path.join(ref, "data", f"sample{n}.gr")):
            continue
        key = f"sample{n}.part.{k}"
        ids[key] = np.array([int(x) for x in open(path).read().split()], dtype=np.uint32)
        out["partitions"][key] = {"sample": f"sample{n}", "parts": k, "n": int(ids[key].size),
                                  "source": f"src/{base}"}
    with open(os.path.join(HERE, "metis_golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "metis_partitions.npz"), **ids)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SCC_REFERENCE_DIR", "/root/reference"))
