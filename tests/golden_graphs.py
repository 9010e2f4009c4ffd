"""Small graphs with known structure used by the CPU and GPU parity tests."""
import numpy as np

from oracle.gtgraph_ref import build_csr


def csr(V, arcs):
    arcs = np.asarray(arcs, dtype=np.int64).reshape(-1, 2)
    Fr, Fc, Br, Bc = build_csr(V, arcs[:, 0], arcs[:, 1])
    return V, Fr, Fc, Br, Bc


def edge_cases():
    """(name, V, src, dst) covering the cases the drivers branch on."""
    rng = np.random.default_rng(7)
    cases = []
    cases.append(("single_vertex", 1, [], []))
    cases.append(("isolated_10", 10, [], []))
    cases.append(("self_loop_only", 3, [1, 2], [1, 2]))
    cases.append(("two_cycle", 2, [1, 2], [2, 1]))
    cases.append(("two_cycle_dup", 2, [1, 2, 1], [2, 1, 2]))
    cases.append(("two_cycles_chain", 6, [1, 2, 2, 3, 4, 4, 5, 6], [2, 1, 3, 4, 3, 5, 6, 5]))
    cases.append(("dag_chain_100", 100, list(range(1, 100)), list(range(2, 101))))
    cases.append(("rev_chain_100", 100, list(range(2, 101)), list(range(1, 100))))
    cases.append(("cycle_257", 257, list(range(1, 258)), list(range(2, 258)) + [1]))
    # star: hub with degree above the heavy-vertex threshold
    n = 2000
    hub_s = [1] * (n - 1) + list(range(2, n + 1))
    hub_d = list(range(2, n + 1)) + [1] * (n - 1)
    cases.append(("bistar_2000", n, hub_s, hub_d))
    cases.append(("out_star_2000", n, [1] * (n - 1), list(range(2, n + 1))))
    # many 2-cycles hanging off a cycle (trim-2 heavy)
    s, d = list(range(1, 51)), list(range(2, 51)) + [1]
    for k in range(51, 151, 2):
        s += [k, k + 1, k]
        d += [k + 1, k, 1 + (k % 50)]
    cases.append(("two_cycles_on_ring", 150, s, d))
    # random graphs of several densities
    for i, (V, m) in enumerate([(50, 60), (200, 400), (500, 2500), (3000, 4000), (3000, 12000)]):
        cases.append((f"random_{V}_{m}", V, rng.integers(1, V + 1, m).tolist(), rng.integers(1, V + 1, m).tolist()))
    # planted SCC chain with duplicates and self loops
    V = 400
    s, d = [], []
    for b in range(8):
        blk = list(range(1 + 50 * b, 51 + 50 * b))
        s += blk
        d += blk[1:] + blk[:1]
        s += blk[:10]
        d += blk[:10]  # self loops
        if b < 7:
            s += [blk[3]] * 2
            d += [blk[-1] + 7] * 2  # duplicated link to the next block
    cases.append(("planted_chain_400", V, s, d))
    return cases
