"""scc_run_async + scc_finish: the same labels, counters and status as the
synchronous scc_run, runs queued back to back on one stream, device-side
errors reported by scc_finish, host inputs refused."""
import ctypes

import numpy as np
import pytest

import detectingscc_b200 as scc
from detectingscc_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = scc.Engine(0)
    yield e
    e.close()


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _graphs():
    from detectingscc_b200 import graphs
    V, s, d = graphs.rmat(16, seed=4)                       # whole-GPU path
    yield "rmat16", scc.graph_from_arcs(V, s.numpy(), d.numpy())
    V, s, d = graphs.planted_random(seed=3)                 # single-CTA path
    yield "planted", scc.graph_from_arcs(V, s.numpy(), d.numpy())


@pytest.mark.parametrize("algo,w", [("h", 1), ("g", 1), ("y", 8)])
def test_async_equals_sync(engine, oracle_lib, algo, w):
    import torch
    for name, g in _graphs():
        t = [_dev(a) for a in (g.Fr, g.Fc, g.Br, g.Bc)]
        a_out = torch.empty(g.V, dtype=torch.int32, device="cuda")
        b_out = torch.empty(g.V, dtype=torch.int32, device="cuda")
        a = engine.run_device(g.V, g.E, *t, labels_out=a_out, algo=algo, warp=w)
        assert engine.run_device(g.V, g.E, *t, labels_out=b_out, algo=algo, warp=w, wait=False) is None
        b = engine.finish()
        assert torch.equal(a_out, b_out), (name, algo)
        assert (a.num_sccs, a.num_trim1, a.num_trim2, a.num_pivot) == (b.num_sccs, b.num_trim1, b.num_trim2,
                                                                        b.num_pivot), (name, algo)
        assert b.stats["kernel_ms"] > 0 and b.stats["used_block_path"] == a.stats["used_block_path"]
        lab, n = oracle_lib.tarjan(g.V, g.Fr, g.Fc)
        assert np.array_equal(b_out.cpu().numpy().view(np.uint32), lab[1:]) and b.num_sccs == n


def test_async_runs_back_to_back(engine):
    """Three runs queued on one stream without waiting: each one's labels are
    complete in stream order; finish reports the last."""
    import torch
    gs = [g for _, g in _graphs()]
    outs, keep = [], []
    for g in gs + gs[:1]:
        t = [_dev(a) for a in (g.Fr, g.Fc, g.Br, g.Bc)]
        o = torch.empty(g.V, dtype=torch.int32, device="cuda")
        engine.run_device(g.V, g.E, *t, labels_out=o, algo="h", wait=False)
        outs.append(o)
        keep.append(t)                                          # inputs alive until the runs are done
    last = engine.finish()
    assert engine.finish().num_sccs == 0                      # nothing pending any more
    for g, o in zip(gs + gs[:1], outs):
        assert np.array_equal(o.cpu().numpy().view(np.uint32), engine.run(g, algo="h").labels)
    assert last.num_sccs == engine.run(gs[0], algo="h").num_sccs


def test_async_errors(engine):
    import torch
    g = scc.graph_from_arcs(6, np.array([1, 2, 3, 4, 5, 6]), np.array([2, 3, 1, 5, 6, 4]))
    fc = g.Fc.copy()
    fc[2] = 9                                                   # an id above V: found on the device
    t = [_dev(a) for a in (g.Fr, fc, g.Br, g.Bc)]
    o = torch.empty(6, dtype=torch.int32, device="cuda")
    engine.run_device(6, 6, *t, labels_out=o, algo="h", wait=False)
    with pytest.raises(scc.SCCError) as e:
        engine.finish()
    assert e.value.code == 23
    # host inputs cannot be left running: refused
    view = N.CsrView(g.V, g.E, g.Fr.ctypes.data, g.Fc.ctypes.data, g.Br.ctypes.data, g.Bc.ctypes.data)
    lib = N.lib()
    assert lib.scc_run_async(engine._h, ctypes.byref(view), ord("h"), 3, 1, None, None) == 1
    # the context works afterwards
    assert engine.run(g, algo="h").num_sccs == 2
