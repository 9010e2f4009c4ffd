"""The product GTgraph loader against the restated reference loader."""
import os

import numpy as np
import pytest

import detectingscc_b200 as scc
from conftest import SAMPLES
from oracle.gtgraph_ref import build_csr, load_gtgraph, write_gtgraph


@pytest.mark.parametrize("name", SAMPLES)
def test_loader_matches_reference_layout(golden, native, tmp_path, name):
    z = golden[name]
    V = int(z["V"])
    path = str(tmp_path / f"{name}.gr")
    write_gtgraph(path, V, z["src"], z["dst"], name)
    g = scc.load_graph(path)
    V2, E2, Fr, Fc, Br, Bc = load_gtgraph(path)
    assert (g.V, g.E) == (V2, E2) == (V, int(z["E"]))
    for a, b in ((g.Fr, Fr), (g.Fc, Fc), (g.Br, Br), (g.Bc, Bc)):
        assert np.array_equal(a, b)
    assert g.Fr[0] == 0 and g.Fr[1] == 0 and g.Fr[V + 1] == g.E


def test_loadFullGraph_mirror(golden, native, tmp_path):
    z = golden["sample4"]
    path = str(tmp_path / "s4.gr")
    write_gtgraph(path, int(z["V"]), z["src"], z["dst"])
    CSize, RSize, Fc, Fr, Bc, Br, Pr = scc.loadFullGraph(path)
    assert (CSize, RSize) == (13, 8)
    assert Fr.shape == (10,) and Br.shape == (10,) and Pr.shape == (10,) and not Pr.any()


def test_binary_roundtrip(golden, native, tmp_path):
    z = golden["sample2"]
    g = scc.graph_from_arcs(int(z["V"]), z["src"], z["dst"])
    p = str(tmp_path / "g.bin")
    scc.save_binary(p, g)
    h = scc.load_graph(p)
    for k in ("Fr", "Fc", "Br", "Bc"):
        assert np.array_equal(getattr(g, k), getattr(h, k))


def test_graph_from_arcs_matches_builder(native):
    rng = np.random.default_rng(0)
    V = 777
    s, d = rng.integers(1, V + 1, 5000), rng.integers(1, V + 1, 5000)
    g = scc.graph_from_arcs(V, s, d)
    Fr, Fc, Br, Bc = build_csr(V, s, d)
    for a, b in ((g.Fr, Fr), (g.Fc, Fc), (g.Br, Br), (g.Bc, Bc)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("body,code", [
    ("p sp 3 2\na 1 2 1\n", "SCC_ERR_BAD_GRAPH"),          # fewer arcs than declared
    ("p sp 3 1\na 1 4 1\n", "SCC_ERR_BAD_GRAPH"),          # id above V
    ("p sp 3 1\na 0 2 1\n", "SCC_ERR_BAD_GRAPH"),          # id 0
    ("p sp\n", "SCC_ERR_BAD_GRAPH"),                       # truncated header
])
def test_malformed_files_are_reported(native, tmp_path, body, code):
    p = str(tmp_path / "bad.gr")
    with open(p, "w") as f:
        f.write("c\n" * 7 + body)
    with pytest.raises(scc.SCCError) as e:
        scc.load_graph(p)
    assert code in str(e.value)


def test_missing_file(native, tmp_path):
    with pytest.raises(scc.SCCError) as e:
        scc.load_graph(str(tmp_path / "nope.gr"))
    assert "SCC_ERR_IO" in str(e.value)


def test_save_gtgraph_roundtrip(native, tmp_path):
    """The library's GTgraph writer produces what the reference loader
    (restated) and the product loader read back as the same graph."""
    rng = np.random.default_rng(4)
    V = 1000
    s, d = rng.integers(1, V + 1, 7000), rng.integers(1, V + 1, 7000)
    g = scc.graph_from_arcs(V, s, d)
    p = str(tmp_path / "w.gr")
    scc.save_gtgraph(p, g)
    V2, E2, Fr, Fc, Br, Bc = load_gtgraph(p)
    h = scc.load_graph(p)
    assert (V2, E2) == (g.V, g.E) == (h.V, h.E)
    for k, ref in zip(("Fr", "Fc", "Br", "Bc"), (Fr, Fc, Br, Bc)):
        assert np.array_equal(getattr(g, k), ref) and np.array_equal(getattr(h, k), ref), k
