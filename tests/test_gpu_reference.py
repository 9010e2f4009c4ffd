"""Parity with the reference's own CUDA code, run on the B200.

oracle/_ref/scc_ref is the reference's unchanged scc.cu, scc_kernels.cu,
scc_WCC.cu and scc_Coloring.cu built for sm_100a and linked with a
project-written loader (oracle/Makefile).  The reference prints counts only,
so parity is on "Number Of Sccs" and on vHong's "numberOf1Sccs"; labels are
pinned against Tarjan in test_gpu_parity.py.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, SAMPLES

pytestmark = pytest.mark.gpu
REF = os.path.join(ROOT, "oracle", "_ref", "scc_ref")
LINKED = os.path.join(ROOT, "oracle", "_ref", "scc_linked")


def _ref(path, algo, p, q, w):
    out = subprocess.run([REF, "-a", algo, "-p", str(p), "-q", str(q), "-w", str(w), "-f", path],
                         capture_output=True, text=True, timeout=120)
    return out


def _ours(native, path, algo, p, q, w):
    return subprocess.run([native.CLI_PATH, "-a", algo, "-p", str(p), "-q", str(q), "-w", str(w), "-f", path],
                          capture_output=True, text=True, timeout=120)


def _count(text, pat):
    m = re.search(pat, text)
    return int(m.group(1)) if m else None


@pytest.fixture(scope="module")
def gr_files(golden, tmp_path_factory):
    from oracle.gtgraph_ref import write_gtgraph
    d = tmp_path_factory.mktemp("gr")
    paths = {}
    for name in SAMPLES:
        z = golden[name]
        p = str(d / f"{name}.gr")
        write_gtgraph(p, int(z["V"]), z["src"], z["dst"], name)
        paths[name] = p
    return paths


@pytest.mark.skipif(not os.path.exists(REF), reason="reference binary not built (make -C oracle ref)")
@pytest.mark.parametrize("name", SAMPLES)
@pytest.mark.parametrize("algo,p,q,w", [("g", 1, 0, 1), ("x", 1, 0, 8), ("h", 1, 1, 1), ("h", 0, 0, 1),
                                        ("y", 1, 1, 8), ("y", 0, 1, 4)])
def test_counts_match_reference_binary(native, oracle_lib, golden, gr_files, name, algo, p, q, w):
    ref = _ref(gr_files[name], algo, p, q, w)
    ours = _ours(native, gr_files[name], algo, p, q, w)
    assert ref.returncode == 0 and ours.returncode == 0, (ref.stdout, ours.stdout, ours.stderr)
    n_ref = _count(ref.stdout, r"Number Of Sccs : (-?\d+)")
    n_ours = _count(ours.stdout, r"Number Of Sccs : (-?\d+)")
    assert n_ref == n_ours == int(golden[name]["nscc"])
    norm = lambda s: re.sub(r"Time : [0-9.]+", "Time : T", s)  # noqa: E731
    if algo == "g":
        # numberOf1Sccs depends on the first pivot and on the order of the
        # trims; the reference picks the pivot with unsynchronised writes, so
        # its count can differ between its own runs (sample2: 3887 recorded,
        # 3744 seen once).  Ours is deterministic and must equal the
        # reference's recorded output; a live reference run that disagrees
        # is only reported.
        n1 = _count(ours.stdout, r"numberOf1Sccs: (-?\d+)")
        rec = _recorded().get(f"{name}:{algo}:p{p}:q{q}:w{w}")
        if rec is not None and rec.get("numberOf1Sccs") is not None:
            assert n1 == rec["numberOf1Sccs"]
        n1_ref = _count(ref.stdout, r"numberOf1Sccs: (-?\d+)")
        if n1_ref != n1:
            import warnings
            warnings.warn(f"{name}: this run of the reference printed numberOf1Sccs {n1_ref}, ours {n1}")
            return
    # same stdout lines, only the time value differs
    assert norm(ref.stdout) == norm(ours.stdout)


def _recorded():
    import json
    pth = os.path.join(ROOT, "tests", "golden", "ref_counts.json")
    return json.load(open(pth)) if os.path.exists(pth) else {}


@pytest.mark.skipif(not os.path.exists(REF), reason="reference binary not built (make -C oracle ref)")
@pytest.mark.parametrize("name", ["sample128", "sample2"])
def test_hong_trim2_count_at_most_truth(golden, gr_files, name):
    # with -q 1 the reference marks both members of a 2-cycle with
    # unsynchronised byte writes and can lose the trim2 tag: never above truth
    ref = _ref(gr_files[name], "g", 1, 1, 1)
    assert ref.returncode == 0
    assert _count(ref.stdout, r"Number Of Sccs : (-?\d+)") <= int(golden[name]["nscc"])


def test_recorded_reference_counts(golden):
    import json
    p = os.path.join(ROOT, "tests", "golden", "ref_counts.json")
    if not os.path.exists(p):
        pytest.skip("tests/golden/ref_counts.json not recorded yet")
    rec = json.load(open(p))
    for key, r in rec.items():
        name = key.split(":")[0]
        if ":q1:" in key and key.split(":")[1] in "gx":
            assert r["num_sccs"] <= int(golden[name]["nscc"])
        else:
            assert r["num_sccs"] == int(golden[name]["nscc"]), key


@pytest.mark.skipif(not os.path.exists(LINKED), reason="linked drop-in not built (make -C oracle linked)")
@pytest.mark.parametrize("name", SAMPLES)
@pytest.mark.parametrize("algo,p,q,w", [("g", 1, 0, 1), ("g", 1, 1, 1), ("x", 1, 0, 8), ("h", 1, 1, 1),
                                        ("h", 0, 0, 1), ("y", 1, 1, 8), ("y", 0, 1, 4)])
def test_reference_main_linked_against_the_library(native, golden, gr_files, name, algo, p, q, w):
    """The reference's unchanged scc.cu linked against libscc_b200.so (its
    vHong / vSlota / wHong / wSlota / loadFullGraph resolved from the
    library) prints what this project's CLI prints and the SCC count of the
    reference binary and of the fixture's known answer."""
    args = ["-a", algo, "-p", str(p), "-q", str(q), "-w", str(w), "-f", gr_files[name]]
    linked = subprocess.run([LINKED] + args, capture_output=True, text=True, timeout=120)
    ours = _ours(native, gr_files[name], algo, p, q, w)
    assert linked.returncode == 0 and ours.returncode == 0, (linked.stdout, linked.stderr)
    norm = lambda s: re.sub(r"Time : [0-9.]+", "Time : T", s)  # noqa: E731
    assert norm(linked.stdout) == norm(ours.stdout)
    assert _count(linked.stdout, r"Number Of Sccs : (-?\d+)") == int(golden[name]["nscc"])
    if os.path.exists(REF) and not (algo in "gx" and q == 1):   # the reference's Hong -q 1 can under-count
        ref = _ref(gr_files[name], algo, p, q, w)
        assert ref.returncode == 0
        assert _count(ref.stdout, r"Number Of Sccs : (-?\d+)") == _count(linked.stdout, r"Number Of Sccs : (-?\d+)")
