"""The C-ABI library loads and exports every entry point of include/*.h."""
import ctypes
import os
import re

import xpu_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"^\s*(?:int|void|uint32_t)\s+(xpuB200\w+)\s*\(", src, re.M)
    return sorted(set(names))


def test_library_exports_declared_symbols():
    L = xpu_b200.lib()
    names = declared_symbols()
    assert len(names) >= 10
    for n in names:
        assert hasattr(L, n), n


def test_library_is_sm100a_build():
    data = open(xpu_b200.LIB_PATH, "rb").read()
    assert b"sm_100a" in data
