"""The METIS input converter (MetisInput.cpp:12-141) and the partition
reader (load.cpp:115-130), pinned by the reference's own shipped files: for
every sample graph whose converter output the reference ships, the bytes
scc_save_metis and the scc_metis command write must hash to the same
SHA-256 (tests/golden/metis_golden.json, tests/golden/make_metis_golden.py).
"""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import detectingscc_b200 as scc
from conftest import GOLDEN
from oracle.gtgraph_ref import build_csr, write_gtgraph

META = json.load(open(os.path.join(GOLDEN, "metis_golden.json")))
PARTS = np.load(os.path.join(GOLDEN, "metis_partitions.npz"))


def _graph(golden, name):
    z = golden[name]
    V = int(z["V"])
    return scc.Graph(V, len(z["src"]), *build_csr(V, z["src"].astype(np.int64), z["dst"].astype(np.int64)))


@pytest.mark.parametrize("name", sorted(META["converter"]))
def test_converter_matches_reference_output(native, golden, tmp_path, name):
    want = META["converter"][name]
    out = str(tmp_path / "out.graph")
    scc.save_metis(out, _graph(golden, name))
    data = open(out, "rb").read()
    assert len(data) == want["bytes"]
    assert hashlib.sha256(data).hexdigest() == want["sha256"]


@pytest.mark.parametrize("name", ["sample0", "sample128"])
def test_converter_command(native, golden, tmp_path, name):
    z = golden[name]
    gr = str(tmp_path / f"{name}.gr")
    write_gtgraph(gr, int(z["V"]), z["src"], z["dst"], name)
    r = subprocess.run([native.METIS_CLI_PATH, gr], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    data = open(tmp_path / "MeTiSInput1024.graph", "rb").read()     # the reference tool's output name
    assert hashlib.sha256(data).hexdigest() == META["converter"][name]["sha256"]
    r = subprocess.run([native.METIS_CLI_PATH, str(tmp_path / "missing.gr"), "x.graph"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and r.stdout == "Error Reading graph file\n"


@pytest.mark.parametrize("key", sorted(META["partitions"]))
def test_partition_reader(native, golden, tmp_path, key):
    rec = META["partitions"][key]
    ids = PARTS[key].tolist()
    V = int(golden[rec["sample"]]["V"])
    p = tmp_path / "part"
    p.write_text("\n".join(str(x) for x in ids) + "\n")
    Pr = scc.load_partition(str(p), V)
    assert Pr.shape == (V + 2,) and Pr[0] == 0 and Pr[V + 1] == 0
    assert Pr[1:V + 1].tolist() == ids[:V]


def test_partition_reader_errors(native, tmp_path):
    p = tmp_path / "short"
    p.write_text("1 2\n")
    with pytest.raises(scc.SCCError):
        scc.load_partition(str(p), 3)
    with pytest.raises(scc.SCCError):
        scc.load_partition(str(tmp_path / "none"), 3)


def test_loader_reads_partition_from_environment(native, golden, tmp_path, monkeypatch):
    ids = PARTS["sample128.part.10"].tolist()
    z = golden["sample128"]
    gr = str(tmp_path / "s.gr")
    write_gtgraph(gr, int(z["V"]), z["src"], z["dst"], "sample128")
    p = tmp_path / "part"
    p.write_text(" ".join(str(x) for x in ids))
    monkeypatch.setenv("SCC_METIS_PARTITION", str(p))
    *_, Pr = scc.loadFullGraph(gr)
    assert Pr[1:129].tolist() == ids
    monkeypatch.delenv("SCC_METIS_PARTITION")
    *_, Pr = scc.loadFullGraph(gr)
    assert not Pr.any()
