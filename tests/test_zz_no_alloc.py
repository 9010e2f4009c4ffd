"""scc_run_noalloc: the entry point for callers that cannot allocate device
memory (their GPU memory is reserved up front by another allocator, or their
host forbids allocations outside its own pool).  It must give exactly the
labels and counts of scc_run (integer labels: tolerance 0), call after call,
using only its built-in scratch array.

Collected last on purpose (file name), so a failure here does not hide the
rest of the suite; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _view(native, V, E, Fr, Fc, Br, Bc):
    return native.CsrView(V, E, Fr.data_ptr(), Fc.data_ptr(), Br.data_ptr(), Bc.data_ptr())


def _noalloc(native, view, algo, flags, warp, out, stream):
    st = native.Stats()
    rc = native.lib().scc_run_noalloc(ctypes.byref(view), ord(algo), flags | native.FLAG_DEVICE, warp,
                                      out.data_ptr(), ctypes.byref(st), stream)
    return rc, st


@pytest.mark.parametrize("algo,warp", [("h", 1), ("g", 1), ("y", 8), ("x", 4)])
def test_noalloc_matches_scc_run_twice(native, algo, warp):
    import torch

    import detectingscc_b200 as scc
    from detectingscc_b200 import graphs
    V, s, d = graphs.rmat(12, seed=4, device="cuda")
    Fr, Fc, Br, Bc = graphs.csr_from_arcs_torch(V, s, d)
    E = int(Fc.shape[0])
    assert V <= 16384 and E <= 262144
    stream = torch.cuda.current_stream().cuda_stream
    flags = native.FLAG_TRIM1 | native.FLAG_TRIM2

    eng = scc.Engine(0)
    try:
        ref = torch.empty(V, dtype=torch.int32, device="cuda")
        r = eng.run_device(V, E, Fr, Fc, Br, Bc, labels_out=ref, algo=algo, warp=warp)
    finally:
        eng.close()
    view = _view(native, V, E, Fr, Fc, Br, Bc)
    for _ in range(2):  # the scratch keeps the previous call's contents
        out = torch.full((V,), -1, dtype=torch.int32, device="cuda")
        rc, st = _noalloc(native, view, algo, flags, warp, out, stream)
        assert rc == 0, native.status_string(rc)
        assert torch.equal(out, ref)
        assert (st.num_sccs, st.num_trim1, st.num_trim2, st.num_pivot) == \
            (r.num_sccs, r.num_trim1, r.num_trim2, r.num_pivot)


def test_noalloc_other_graph_after_a_bigger_one(native):
    import torch

    import detectingscc_b200 as scc
    from detectingscc_b200 import graphs
    stream = torch.cuda.current_stream().cuda_stream
    for gen in (lambda: graphs.grid(120, seed=2, device="cuda"), lambda: graphs.planted_random(seed=5, device="cuda")):
        V, s, d = gen()
        Fr, Fc, Br, Bc = graphs.csr_from_arcs_torch(V, s, d)
        E = int(Fc.shape[0])
        eng = scc.Engine(0)
        try:
            ref = torch.empty(V, dtype=torch.int32, device="cuda")
            eng.run_device(V, E, Fr, Fc, Br, Bc, labels_out=ref, algo="h")
        finally:
            eng.close()
        out = torch.empty(V, dtype=torch.int32, device="cuda")
        rc, _ = _noalloc(native, _view(native, V, E, Fr, Fc, Br, Bc), "h", native.FLAG_TRIM1, 1, out, stream)
        assert rc == 0 and torch.equal(out, ref)


def test_noalloc_rejects_graphs_above_its_limit(native):
    import torch
    V, E = 16385, 10
    Fr = torch.zeros(V + 2, dtype=torch.int32, device="cuda")
    Fc = torch.ones(E, dtype=torch.int32, device="cuda")
    out = torch.empty(V, dtype=torch.int32, device="cuda")
    view = _view(native, V, E, Fr, Fc, Fr, Fc)
    rc, _ = _noalloc(native, view, "h", 0, 1, out, None)
    assert rc == 4  # SCC_ERR_TOO_LARGE, before anything runs
    # without SCC_FLAG_DEVICE the inputs would have to be copied: refused
    small = _view(native, 3, E, Fr, Fc, Fr, Fc)
    rc = native.lib().scc_run_noalloc(ctypes.byref(small), ord("h"), 0, 1, out.data_ptr(), None, None)
    assert rc == 1  # SCC_ERR_INVALID_ARG


def test_noalloc_at_its_exact_limit_matches_tarjan(native, oracle_lib):
    """A graph of exactly SCC_NOALLOC_MAX_VERTICES vertices and
    SCC_NOALLOC_MAX_EDGES arcs (duplicates kept) fits the built-in scratch
    array: labels equal Tarjan's and scc_run's, twice in a row."""
    import torch

    import detectingscc_b200 as scc
    V, E = 16384, 262144
    rng = np.random.default_rng(17)
    # uniform arcs, mean out-degree 16: one giant SCC plus trimmed vertices
    src = rng.integers(1, V + 1, E)
    dst = rng.integers(1, V + 1, E)
    g = scc.graph_from_arcs(V, src, dst)
    assert (g.V, g.E) == (V, E)
    lab, n = oracle_lib.tarjan(g.V, g.Fr, g.Fc)
    dev = [torch.from_numpy(a.view(np.int32)).cuda() for a in (g.Fr, g.Fc, g.Br, g.Bc)]
    stream = torch.cuda.current_stream().cuda_stream
    view = _view(native, V, E, *dev)
    eng = scc.Engine(0)
    try:
        ref = torch.empty(V, dtype=torch.int32, device="cuda")
        r = eng.run_device(V, E, *dev, labels_out=ref, algo="h")
    finally:
        eng.close()
    assert r.num_sccs == n
    for algo in ("h", "g"):
        for _ in range(2):
            out = torch.full((V,), -1, dtype=torch.int32, device="cuda")
            rc, st = _noalloc(native, view, algo, native.FLAG_TRIM1 | native.FLAG_TRIM2, 1, out, stream)
            assert rc == 0, native.status_string(rc)
            assert st.num_sccs == n
            got = out.cpu().numpy().view(np.uint32)
            assert np.array_equal(got, lab[1:])
            if algo == "h":
                assert torch.equal(out, ref)


def test_noalloc_rejects_flags_it_does_not_use(native):
    import torch
    V, E = 4, 2
    Fr = torch.tensor([0, 0, 1, 2, 2, 2], dtype=torch.int32, device="cuda")
    Fc = torch.tensor([2, 3], dtype=torch.int32, device="cuda")
    out = torch.empty(V, dtype=torch.int32, device="cuda")
    view = _view(native, V, E, Fr, Fc, Fr, Fc)
    for extra in (native.FLAG_DERIVE_REVERSE, native.FLAG_FORCE_GRID, native.FLAG_INSTRUMENT):
        rc, _ = _noalloc(native, view, "h", extra, 1, out, None)
        assert rc == 1  # SCC_ERR_INVALID_ARG
