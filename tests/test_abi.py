"""The C-ABI library loads and exports every symbol include/*.h declares."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import REFERENCE_DIR, ROOT


def _declared_c_functions():
    names = []
    for h in ("scc_b200.h",):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:int|void|const char \*)\s*\**\s*(scc_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported(native):
    lib = native.lib()
    declared = _declared_c_functions()
    assert set(declared) == set(native.C_SYMBOLS), declared
    for name in declared:
        assert hasattr(lib, name), name
    out = subprocess.check_output(["nm", "-D", "--defined-only", native.LIB_PATH]).decode()
    for sym in native.CXX_SYMBOLS:
        assert re.search(rf"\bT {sym}\b", out), sym


def test_compat_header_matches_mangled_names(native):
    text = open(os.path.join(ROOT, "include", "scc_compat.h")).read()
    for sym in native.CXX_SYMBOLS:
        assert sym in text


def test_status_strings_and_version(native):
    lib = native.lib()
    assert b"sm_100a" in lib.scc_version()
    for code in native.STATUS_NAMES:
        assert native.status_string(code) != "unknown status"


def test_no_gpu_is_an_error_not_a_crash(native):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = native.lib().scc_create(0, ctypes.byref(h))
    assert rc == 5  # SCC_ERR_NO_DEVICE


def test_python_mirror_fails_loudly_without_library(native, monkeypatch):
    from detectingscc_b200 import _native
    monkeypatch.setattr(_native, "_lib", None)
    monkeypatch.setattr(_native, "LIB_PATH", "/nonexistent/libscc_b200.so")
    with pytest.raises(_native.NativeLibraryError):
        _native.lib()


def test_reference_main_links_against_the_library(native, tmp_path):
    """The reference's own scc.cu (unchanged, compiled from the reference
    checkout where present) links against libscc_b200.so in place of its
    scc_kernels / scc_WCC / scc_Coloring / load objects."""
    ref = REFERENCE_DIR
    if not os.path.isdir(os.path.join(ref, "src")):
        pytest.skip("reference checkout not present")
    out = str(tmp_path / "scc_linked")
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-I" + os.path.join(ref, "include"),
           os.path.join(ref, "src", "scc.cu"), "-L" + os.path.dirname(native.LIB_PATH), "-lscc_b200",
           "-Xlinker", "-rpath=" + os.path.dirname(native.LIB_PATH), "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    nm = subprocess.check_output(["nm", "-u", out]).decode()
    for sym in ("_Z5vHongjjPjS_S_S_bb", "_Z6vSlotajjPjS_S_S_bb", "_Z13loadFullGraphPKcPjS1_PS1_S2_S2_S2_S2_"):
        assert sym in nm      # resolved from the library at run time
    # running it without arguments prints the reference's help (no GPU needed)
    r = subprocess.run([out], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and r.stdout.startswith("To execute:")
