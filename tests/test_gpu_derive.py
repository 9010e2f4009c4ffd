"""Reverse CSR built on the device (scc_derive_reverse, SCC_FLAG_DERIVE_REVERSE):
bit-exact against the host loader's reverse CSR (same layout, in-lists in
ascending source order), the same labels with and without it, and
malformed forward CSRs answered with SCC_ERR_BAD_GRAPH."""
import numpy as np
import pytest

import detectingscc_b200 as scc
from conftest import SAMPLES
from golden_graphs import edge_cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = scc.Engine(0)
    yield e
    e.close()


def _cases(golden):
    from detectingscc_b200 import graphs
    out = [(n, V, s, d) for n, V, s, d in edge_cases()]
    for n in SAMPLES:
        z = golden[n]
        out.append((n, int(z["V"]), z["src"], z["dst"]))
    rng = np.random.default_rng(3)
    out.append(("random_dups_loops", 500, rng.integers(1, 501, 6000), rng.integers(1, 501, 6000)))
    V, s, d = graphs.rmat(12, seed=5, clean=False)          # hubs with long in-lists, self-loops, duplicates
    out.append(("rmat12_raw", V, s.numpy(), d.numpy()))
    # in-lists longer than one shared-memory chunk (4,096): sorted chunks, then merge passes
    for n in (4097, 9000, 20000):
        src = rng.permutation(np.arange(2, n + 2))
        src = np.concatenate([src, src[:100]])              # duplicate arcs into the hub
        out.append((f"hub_in_{n}", n + 1, src, np.ones(src.size, np.int64)))
    return out


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def test_reverse_csr_bit_exact(engine, golden):
    import torch
    for name, V, s, d in _cases(golden):
        g = scc.graph_from_arcs(V, np.asarray(s), np.asarray(d))
        Br = torch.full((V + 2,), -1, dtype=torch.int32, device="cuda")
        Bc = torch.full((max(g.E, 1),), -1, dtype=torch.int32, device="cuda")
        engine.derive_reverse(V, g.E, _dev(g.Fr), _dev(g.Fc) if g.E else Bc, Br, Bc)
        torch.cuda.synchronize()
        assert np.array_equal(Br.cpu().numpy().view(np.uint32), g.Br), name
        assert np.array_equal(Bc.cpu().numpy().view(np.uint32)[:g.E], g.Bc), name


@pytest.mark.parametrize("algo,w", [("g", 1), ("h", 1), ("y", 8)])
def test_same_labels_with_derived_reverse(engine, golden, algo, w):
    import torch
    for name, V, s, d in _cases(golden):
        g = scc.graph_from_arcs(V, np.asarray(s), np.asarray(d))
        a = engine.run(g, algo=algo, warp=w)
        b = engine.run(g, algo=algo, warp=w, derive_reverse=True)
        assert np.array_equal(a.labels, b.labels), (name, algo)
        assert (a.num_sccs, a.num_trim1, a.num_trim2, a.num_pivot) == (b.num_sccs, b.num_trim1, b.num_trim2,
                                                                        b.num_pivot), name
        lab = torch.empty(max(V, 1), dtype=torch.int32, device="cuda")
        c = engine.run_device(V, g.E, _dev(g.Fr), _dev(g.Fc) if g.E else lab, None, None, lab, algo=algo, warp=w,
                              derive_reverse=True)
        torch.cuda.synchronize()
        assert c.num_sccs == a.num_sccs, name
        assert np.array_equal(lab.cpu().numpy().view(np.uint32)[:V], a.labels), name


def test_bad_forward_csr_is_rejected(engine):
    import torch
    g = scc.graph_from_arcs(6, np.array([1, 2, 3, 4, 5, 6]), np.array([2, 3, 1, 5, 6, 4]))
    Br = torch.zeros(8, dtype=torch.int32, device="cuda")
    Bc = torch.zeros(6, dtype=torch.int32, device="cuda")
    for bad_fc in ([2, 3, 1, 5, 6, 7], [2, 3, 0, 5, 6, 4]):      # an id above V, an id 0
        fc = np.array(bad_fc, dtype=np.uint32)
        with pytest.raises(scc.SCCError) as ei:
            engine.derive_reverse(6, 6, _dev(g.Fr), _dev(fc), Br, Bc)
        assert ei.value.code == 23
        h = scc.Graph(6, 6, g.Fr, fc, g.Br, g.Bc)
        with pytest.raises(scc.SCCError) as ei:
            engine.run(h, algo="h", derive_reverse=True)
        assert ei.value.code == 23
    fr = g.Fr.copy()
    fr[3], fr[4] = fr[4] + 1, fr[3]                               # offsets going down
    with pytest.raises(scc.SCCError) as ei:
        engine.derive_reverse(6, 6, _dev(fr), _dev(g.Fc), Br, Bc)
    assert ei.value.code == 23
    # the context still works afterwards
    assert engine.run(g, algo="h", derive_reverse=True).num_sccs == 2


def test_host_upload_in_pieces(engine, oracle_lib):
    """R-MAT scale 20 (raw: hubs, duplicates, self-loops) from host memory with
    the reverse CSR built on the device: the forward targets cross in eight
    pieces beside the first kernels of the build; labels equal Tarjan's and
    the run that copies both CSRs."""
    from detectingscc_b200 import graphs
    V, s, d = graphs.rmat(20, seed=9, clean=False)
    g = scc.graph_from_arcs(V, s.numpy(), d.numpy())
    assert (g.E + 4095) // 4096 >= 8 * 512                       # 4,096-arc tiles for eight 512-tile pieces
    for algo in ("h", "g"):
        a = engine.run(g, algo=algo, derive_reverse=True)
        b = engine.run(g, algo=algo)
        lab, n = oracle_lib.tarjan(V, g.Fr, g.Fc)
        assert np.array_equal(a.labels, lab[1:]) and a.num_sccs == n, algo
        assert np.array_equal(a.labels, b.labels), algo
