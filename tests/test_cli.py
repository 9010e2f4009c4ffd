"""The drop-in ./scc command line: argument handling (no GPU needed)."""
import subprocess

import pytest

HELP = (
    "To execute:\n"
    "./scc -a [g/h/x/y/d] -p [0/1] -q [0/1] -w [1/2/4/8/16/32] -f <file>\n"
    "-a algorith to use   g - vHong, h - vSlota, x - wHong, y - wSlota, d - detectSCC\n"
    "-p Trim-1 enable\n-q Trim-2 enable\n-w warp size\n-f input file\n"
    "Please note that the input graph must be in GTgraph format\n"
    "If not provided the results are undefined\n")


def _run(native, *args):
    return subprocess.run([native.CLI_PATH, *args], capture_output=True, text=True, timeout=60)


def test_too_few_arguments_prints_help(native):
    r = _run(native, "-a", "g")
    assert r.returncode == 1 and r.stdout == HELP


def test_detect_scc_reads_its_graph_and_partition_first(native, tmp_path, monkeypatch):
    # -a d (detectSCC) loads the graph, then the METIS partition named by
    # SCC_METIS_PARTITION; a file that cannot be read is reported before any
    # device work, with the reference's messages (load.cpp:24-28, :119-123)
    r = _run(native, "-a", "d", "-p", "1", "-q", "1", "-w", "1", "-f", str(tmp_path / "x.gr"))
    assert r.returncode == 1 and r.stdout.startswith("Error Reading graph file")
    from oracle.gtgraph_ref import write_gtgraph
    gr = str(tmp_path / "g.gr")
    write_gtgraph(gr, 3, [1, 2], [2, 3], "g")
    monkeypatch.setenv("SCC_METIS_PARTITION", str(tmp_path / "missing.part"))
    r = _run(native, "-a", "d", "-p", "1", "-q", "1", "-w", "1", "-f", gr)
    assert r.returncode == 1 and r.stdout.startswith("Error Reading metis graph file")


def test_bad_warp_width_rejected(native, tmp_path):
    r = _run(native, "-a", "y", "-p", "1", "-q", "1", "-w", "3", "-f", str(tmp_path / "x.gr"))
    assert r.returncode == 1


def test_unknown_algorithm_prints_help(native, tmp_path):
    r = _run(native, "-a", "z", "-p", "1", "-q", "1", "-w", "1", "-f", str(tmp_path / "x.gr"))
    assert r.returncode == 1 and r.stdout == HELP


def test_unreadable_graph(native, tmp_path):
    r = _run(native, "-a", "g", "-p", "1", "-q", "1", "-w", "1", "-f", str(tmp_path / "missing.gr"))
    assert r.returncode == 1 and r.stdout.startswith("Error Reading graph file")
