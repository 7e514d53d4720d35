"""The C-ABI library loads and exports every entry point declared in
include/quill_b200.h (no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    out = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            out |= set(re.findall(r"\b(qp_[a-z_0-9]+)\s*\(", src))
    return out


def test_library_exports_header():
    from quill_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    syms = declared_symbols()
    assert len(syms) >= 15
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_create_error_without_device():
    from quill_b200 import api
    lib = api.load_library()
    assert lib.qp_version().decode().startswith("quill_b200")
    # a bad configuration is refused before any device work
    p = api.Params()
    p.nx = p.ny = p.nz = 3
    h = ctypes.c_void_p()
    r = lib.qp_create(ctypes.byref(p), ctypes.byref(h))
    assert r == 1 and b"grid" in lib.qp_last_error(None)
