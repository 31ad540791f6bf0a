"""The C-ABI library loads and exports every symbol include/curegot_b200.h declares."""
import os
import re

import curegot_backward_b200 as cg
from curegot_backward_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "curegot_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cg_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    L = _native.lib()
    names = declared_symbols()
    assert names, "no declarations found"
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_symbols()) <= set(_native.SIGNATURES)


def test_version_and_error_strings():
    L = _native.lib()
    assert b"sm_100a" in L.cg_version()
    assert L.cg_last_error() is not None


def test_namespaces():
    assert callable(cg.numpy.sinkhorn_bcd)
    assert callable(cg.torch.sinkhorn_bcd)
