"""The C-ABI libraries load and export every entry point their headers declare (CPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sparsedirectsolver.jl_b200")


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:sdsb200|sdsa)_[a-z_]+)\s*\(", text)))


@pytest.mark.parametrize("header,lib", [("sdsb200.h", "libsdsb200.so"),
                                        ("sdsb200_analysis.h", "libsdsb200_analysis.so")])
def test_exports(header, lib):
    path = os.path.join(PKG, lib)
    if not os.path.exists(path):
        pytest.fail(f"{lib} is not built (run __graft_entry__.build())")
    so = ctypes.CDLL(path)
    names = declared(header)
    assert len(names) >= 5
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    import sys
    sys.path.insert(0, PKG)
    from sdsb200 import capi
    assert set(capi.EXPORTS) == set(declared("sdsb200.h"))
