"""The C-ABI libraries load and export every entry point their header
declares (no GPU needed: nothing is called)."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "pllcart3d_gpu.h")


def declared(prefix):
    txt = open(HDR).read()
    # drop comments
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(" + prefix + r"[a-z0-9_]+)\s*\(", txt)))


def test_pllgpu_symbols_exported():
    from pllcart3d_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        from pllcart3d_b200 import build

        build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared("pllgpu_")
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.EXPORTED_SYMBOLS)
