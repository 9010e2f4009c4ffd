"""detectSCC (-a d, the reference's METIS-partitioned driver) on the B200.

Its printed count is not always the SCC count (range values that coincide
count once), so parity is with what the reference itself prints: the
restated driver in the oracle (pinned on the CPU against the reference
binary's recorded outputs, tests/golden/ref_detect.json) and those recorded
outputs directly, through the CLI and through the reference's own scc.cu
linked against the library.  Integer counts: tolerance 0.
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import detectingscc_b200 as scc
from conftest import GOLDEN, ROOT, SAMPLES
from oracle.gtgraph_ref import build_csr, write_gtgraph

pytestmark = pytest.mark.gpu
REC = json.load(open(os.path.join(GOLDEN, "ref_detect.json")))
PARTS = np.load(os.path.join(GOLDEN, "metis_partitions.npz"))
LINKED = os.path.join(ROOT, "oracle", "_ref", "scc_linked")


@pytest.fixture(scope="module")
def engine():
    e = scc.Engine(0)
    yield e
    e.close()


def _graph(golden, name):
    z = golden[name]
    V = int(z["V"])
    return scc.Graph(V, len(z["src"]), *build_csr(V, z["src"].astype(np.int64), z["dst"].astype(np.int64)))


def _pr(V, part):
    Pr = np.zeros(V + 2, np.uint32)
    if part != "none":
        Pr[1:V + 1] = PARTS[part][:V]
    return Pr


def _check(engine, oracle_lib, g, Pr, t1, t2):
    got = engine.detect(g, Pr, t1=t1, t2=t2)
    counts, rounds, nospace = oracle_lib.detect(g.V, g.Fr, g.Fc, g.Br, g.Bc, Pr, t1, t2)
    assert [got["num_trim1"], got["num_trim2"], got["num_ranges"]] == counts
    assert got["num_sccs"] == sum(counts)
    assert (got["merge_rounds"], got["nospace_mask"]) == (rounds, nospace)
    return got


@pytest.mark.parametrize("key", sorted(REC))
def test_engine_matches_restatement_and_recorded_reference(engine, oracle_lib, golden, key):
    name, part, q = key.split(":")
    g = _graph(golden, name)
    got = _check(engine, oracle_lib, g, _pr(g.V, part), True, q == "q1")
    assert got["num_sccs"] == REC[key]["num_sccs"]


@pytest.mark.parametrize("key", sorted(REC))
def test_cli_and_linked_reference_main_print_what_the_reference_printed(native, golden, tmp_path, key):
    name, part, q = key.split(":")
    z = golden[name]
    gr = str(tmp_path / f"{name}.gr")
    write_gtgraph(gr, int(z["V"]), z["src"], z["dst"], name)
    env = dict(os.environ)
    env.pop("SCC_METIS_PARTITION", None)
    if part != "none":
        pp = tmp_path / "part"
        pp.write_text("\n".join(str(int(x)) for x in PARTS[part]) + "\n")
        env["SCC_METIS_PARTITION"] = str(pp)
    args = ["-a", "d", "-p", "1", "-q", q[1], "-w", "1", "-f", gr]
    mask = lambda s: re.sub(r"Time : [0-9.]+", "Time : T", s)  # noqa: E731
    for exe in (native.CLI_PATH, LINKED):
        if not os.path.exists(exe):
            continue
        r = subprocess.run([exe] + args, capture_output=True, text=True, timeout=120, env=env)
        assert r.returncode == 0, r.stderr
        assert mask(r.stdout) == REC[key]["runs"][0]["stdout"], exe


@pytest.mark.parametrize("seed", range(6))
def test_random_graphs_and_partitions(engine, oracle_lib, seed):
    rng = np.random.default_rng(seed)
    V = int(rng.integers(20, 400))
    m = int(V * rng.uniform(1.0, 4.0))
    src, dst = rng.integers(1, V + 1, m), rng.integers(1, V + 1, m)
    g = scc.graph_from_arcs(V, src, dst)
    nparts = int(rng.choice([1, 2, 3, 5, 10, 17]))
    Pr = np.zeros(V + 2, np.uint32)
    Pr[1:V + 1] = rng.integers(0, nparts, V)
    for t1, t2 in ((1, 1), (1, 0)):
        _check(engine, oracle_lib, g, Pr, t1, t2)


def test_detect_edge_cases(engine, oracle_lib):
    # no arcs ("No space!" every round: the reference tests crossing edges >= E), a self-loop, a 2-cycle
    for V, s, d in ((5, [], []), (3, [1], [1]), (4, [1, 2, 3], [2, 1, 4])):
        g = scc.graph_from_arcs(V, np.array(s, np.int64), np.array(d, np.int64))
        Pr = np.zeros(V + 2, np.uint32)
        Pr[1:V + 1] = np.arange(V) % 2
        _check(engine, oracle_lib, g, Pr, True, True)
