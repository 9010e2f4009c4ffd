"""The CPU oracle pinned against the golden fixtures (scipy + networkx) and
against scipy on random / edge-case graphs."""
import numpy as np
import pytest

from conftest import SAMPLES
from golden_graphs import csr, edge_cases
from oracle.gtgraph_ref import build_csr


def _scipy_labels(V, Fr, Fc):
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    src = np.repeat(np.arange(1, V + 1), np.diff(Fr.astype(np.int64))[1:V + 1])
    A = sp.coo_matrix((np.ones(len(src)), (src - 1, Fc.astype(np.int64) - 1)), shape=(V, V)).tocsr()
    n, lab = connected_components(A, directed=True, connection="strong")
    mn = np.full(n, V + 1, dtype=np.int64)
    np.minimum.at(mn, lab, np.arange(1, V + 1))
    return mn[lab].astype(np.uint32), n


@pytest.mark.parametrize("name", SAMPLES)
def test_tarjan_matches_golden(golden, oracle_lib, name):
    z = golden[name]
    V = int(z["V"])
    Fr, Fc, Br, Bc = build_csr(V, z["src"].astype(np.int64), z["dst"].astype(np.int64))
    lab, n = oracle_lib.tarjan(V, Fr, Fc)
    assert n == int(z["nscc"])
    assert np.array_equal(lab[1:], z["labels"])


@pytest.mark.parametrize("name", SAMPLES)
@pytest.mark.parametrize("t1", [0, 1])
@pytest.mark.parametrize("t2", [0, 1])
def test_phase_restatements_match_golden(golden, oracle_lib, name, t1, t2):
    z = golden[name]
    V = int(z["V"])
    Fr, Fc, Br, Bc = build_csr(V, z["src"].astype(np.int64), z["dst"].astype(np.int64))
    for fn in (oracle_lib.hong, oracle_lib.slota):
        lab, counts = fn(V, Fr, Fc, Br, Bc, t1, t2)
        assert np.array_equal(lab[1:], z["labels"])
        assert sum(counts) == int(z["nscc"])


def test_known_answer_counts(golden):
    # known answers listed for the reference's own sample graphs
    expect = {"sample0": 4, "sample4": 4, "sample5": 3, "sample1": 3, "sample128": 13, "sample2": 4889}
    for k, v in expect.items():
        assert int(golden[k]["nscc"]) == v
    assert golden["sample0"]["labels"].tolist() == [1, 1, 3, 1, 5, 6]
    assert golden["sample4"]["labels"].tolist() == [1, 2, 2, 1, 1, 2, 7, 8]
    assert golden["sample5"]["labels"].tolist() == [1, 1, 1, 1, 1, 1, 1, 1, 9, 10, 1, 1, 1]


def test_trim_counts_on_sample128(golden, oracle_lib):
    # sample128 has one size-2 SCC: Hong with -q 1 finds it as a trim-2 pair
    z = golden["sample128"]
    V = int(z["V"])
    Fr, Fc, Br, Bc = build_csr(V, z["src"].astype(np.int64), z["dst"].astype(np.int64))
    _, c = oracle_lib.hong(V, Fr, Fc, Br, Bc, 1, 1)
    assert c == [10, 1, 2]
    _, c = oracle_lib.hong(V, Fr, Fc, Br, Bc, 1, 0)
    assert c == [10, 0, 3]


@pytest.mark.parametrize("case", edge_cases(), ids=lambda c: c[0])
def test_oracles_on_edge_cases(oracle_lib, case):
    name, V, s, d = case
    _, Fr, Fc, Br, Bc = csr(V, np.stack([np.asarray(s, np.int64), np.asarray(d, np.int64)], 1) if len(s) else np.zeros((0, 2), np.int64))
    ref, n = _scipy_labels(V, Fr, Fc)
    lab, nt = oracle_lib.tarjan(V, Fr, Fc)
    assert nt == n and np.array_equal(lab[1:], ref)
    for t1 in (0, 1):
        for t2 in (0, 1):
            for fn in (oracle_lib.hong, oracle_lib.slota):
                l2, c = fn(V, Fr, Fc, Br, Bc, t1, t2)
                assert np.array_equal(l2[1:], ref), (name, fn.__name__, t1, t2)
                assert sum(c) == n


def test_generators_vs_scipy(oracle_lib):
    from detectingscc_b200 import graphs
    for gen in (lambda: graphs.planted_random(seed=3), lambda: graphs.rmat(12, seed=5),
                lambda: graphs.grid(48, seed=2)):
        V, s, d = gen()
        g = graphs.to_graph(V, s, d)
        ref, n = _scipy_labels(g.V, g.Fr, g.Fc)
        lab, nt = oracle_lib.tarjan(g.V, g.Fr, g.Fc)
        assert nt == n and np.array_equal(lab[1:], ref)
        lh, ch = oracle_lib.hong(g.V, g.Fr, g.Fc, g.Br, g.Bc, 1, 1)
        ls, cs = oracle_lib.slota(g.V, g.Fr, g.Fc, g.Br, g.Bc, 1, 1)
        assert np.array_equal(lh[1:], ref) and np.array_equal(ls[1:], ref)
        assert sum(ch) == n and sum(cs) == n


def test_planted_oracle_catches_a_wrong_label(oracle_lib):
    # a mistake planted in an oracle output (CPU) is detected by the comparison
    V, Fr, Fc, Br, Bc = csr(4, [[1, 2], [2, 1], [3, 4]])
    lab, n = oracle_lib.tarjan(V, Fr, Fc)
    bad = lab.copy()
    bad[2] = 2
    assert not np.array_equal(bad, lab)
    assert lab[1:].tolist() == [1, 1, 3, 4] and n == 3


def test_oracle_counts_match_recorded_reference_outputs(golden, oracle_lib):
    """tests/golden/ref_counts.json holds the reference binary's own output on
    the fixtures (recorded on a B200 by tests/golden/make_ref_counts.py)."""
    import json
    import os
    from conftest import GOLDEN
    p = os.path.join(GOLDEN, "ref_counts.json")
    if not os.path.exists(p):
        pytest.skip("reference outputs not recorded")
    rec = json.load(open(p))
    for key, r in rec.items():
        name, algo, pp, qq, _ = key.split(":")
        t1, t2 = int(pp[1]), int(qq[1])
        z = golden[name]
        V = int(z["V"])
        Fr, Fc, Br, Bc = build_csr(V, z["src"].astype(np.int64), z["dst"].astype(np.int64))
        fn = oracle_lib.hong if algo in "gx" else oracle_lib.slota
        _, c = fn(V, Fr, Fc, Br, Bc, t1, t2)
        if algo in "gx" and t2:
            assert r["num_sccs"] <= sum(c), key       # the reference can lose a trim-2 tag
        else:
            assert r["num_sccs"] == sum(c), key
        if algo == "g" and not t2:
            assert r["numberOf1Sccs"] == c[0], key


def test_detect_restatement_matches_reference_binary_outputs(oracle_lib, golden):
    """The restated detectSCC (-a d) prints exactly what the reference
    binary printed on the shipped samples with their shipped METIS
    partitions and with none (tests/golden/ref_detect.json, recorded on a
    B200 by tests/golden/make_ref_detect.py; time value masked), including
    the case where its range arithmetic over-counts (sample128, -q 1)."""
    import json
    import os
    from conftest import GOLDEN
    rec = json.load(open(os.path.join(GOLDEN, "ref_detect.json")))
    parts = np.load(os.path.join(GOLDEN, "metis_partitions.npz"))
    assert len(rec) >= 20
    for key, r in rec.items():
        name, part, q = key.split(":")
        z = golden[name]
        V = int(z["V"])
        Fr, Fc, Br, Bc = build_csr(V, z["src"].astype(np.int64), z["dst"].astype(np.int64))
        Pr = np.zeros(V + 2, np.uint32)
        if part != "none":
            Pr[1:V + 1] = parts[part][:V]
        counts, rounds, nospace = oracle_lib.detect(V, Fr, Fc, Br, Bc, Pr, True, q == "q1")
        assert r["stable"]
        assert oracle_lib.detect_stdout(counts, rounds, nospace) == r["runs"][0]["stdout"], key
