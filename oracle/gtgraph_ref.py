"""GTgraph parsing and CSR construction restated from the reference loader.

TEST INFRASTRUCTURE ONLY: the checker for the product loader
(``detectingscc_b200/csrc/gtgraph_load.cpp``) and the source of fixture
graphs.  It follows ``src/load.cpp`` of the reference:

* ``load.cpp:32-33``   skip 7 header lines;
* ``load.cpp:36``      read ``p sp V E``;
* ``load.cpp:42-45``   read exactly E lines ``a u v w`` (w ignored);
* ``load.cpp:47``      sort the pairs by (u, v); duplicates and self-loops stay;
* ``load.cpp:49-77``   1-based forward CSR, ``Fr`` has V+2 entries with
  ``Fr[0] = Fr[1] = 0``;
* ``load.cpp:80-113``  reverse CSR by counting sort; each in-list holds
  sources in ascending order.
"""
from __future__ import annotations

import numpy as np


def parse_gtgraph_text(text: str):
    """Return (V, E, src, dst) as the reference reads them (unsorted)."""
    lines = text.split("\n")
    if len(lines) < 8:
        raise ValueError("GTgraph file too short")
    # load.cpp:32-36 -- seven header lines, then "p sp V E" (whitespace-split)
    rest = "\n".join(lines[7:]).split()
    if len(rest) < 4:
        raise ValueError("missing 'p sp V E' line")
    V = int(rest[2])
    E = int(rest[3])
    toks = rest[4:4 + 4 * E]
    if len(toks) < 4 * E:
        raise ValueError("fewer edge lines than the header declares")
    arr = np.array(toks, dtype=object).reshape(E, 4) if E else np.zeros((0, 4), dtype=object)
    src = np.array([int(x) for x in arr[:, 1]], dtype=np.int64) if E else np.zeros(0, np.int64)
    dst = np.array([int(x) for x in arr[:, 2]], dtype=np.int64) if E else np.zeros(0, np.int64)
    return V, E, src, dst


def build_csr(V: int, src: np.ndarray, dst: np.ndarray):
    """Forward and reverse CSR in the reference's 1-based layout.

    Returns (Fr, Fc, Br, Bc) as uint32 arrays; Fr/Br have V+2 entries.
    """
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    E = src.shape[0]
    if E and (src.min() < 1 or src.max() > V or dst.min() < 1 or dst.max() > V):
        raise ValueError("vertex id outside [1, V]")
    order = np.lexsort((dst, src))          # load.cpp:47, sort by (u, v)
    s = src[order]
    d = dst[order]
    Fr = np.zeros(V + 2, dtype=np.int64)
    np.add.at(Fr, s + 1, 1) if E else None
    Fr = np.cumsum(Fr)
    Fr[0] = 0
    Fc = d.astype(np.uint32)
    # reverse CSR: in-lists ordered by source (load.cpp:103-111 walks the
    # sorted edges in order, so each target's sources come out ascending)
    rorder = np.lexsort((s, d))
    Br = np.zeros(V + 2, dtype=np.int64)
    np.add.at(Br, d + 1, 1) if E else None
    Br = np.cumsum(Br)
    Br[0] = 0
    Bc = s[rorder].astype(np.uint32)
    return Fr.astype(np.uint32), Fc, Br.astype(np.uint32), Bc


def load_gtgraph(path: str):
    with open(path, "r") as f:
        text = f.read()
    V, E, src, dst = parse_gtgraph_text(text)
    Fr, Fc, Br, Bc = build_csr(V, src, dst)
    return V, E, Fr, Fc, Br, Bc


def write_gtgraph(path: str, V: int, src, dst, name: str = "graph") -> None:
    """Write a GTgraph file with the 7-line header the reference skips."""
    src = np.asarray(src)
    dst = np.asarray(dst)
    E = int(src.shape[0])
    with open(path, "w") as f:
        f.write(f"c FILE\t\t\t: {name}\n")
        f.write(f"c No. of vertices\t: {V}\n")
        f.write(f"c No. of directed edges\t: {E}\n")
        f.write("c Max. weight\t\t: 1\n")
        f.write("c Min. weight\t\t: 1\n")
        f.write("c A directed arc from u to v of weight w\n")
        f.write("c is represented below as ' a  u  v  w '\n")
        f.write(f"p sp {V} {E}\n")
        if E:
            lines = np.char.add(np.char.add(np.char.add("a ", src.astype(str)), " "), dst.astype(str))
            f.write("\n".join((lines + " 1").tolist()))
            f.write("\n")
