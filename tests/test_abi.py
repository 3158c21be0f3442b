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


_NOALLOC_OVERFLOW = r"""
import ctypes, sys
sys.path.insert(0, sys.argv[1])
from pllcart3d_b200 import _lib
L = _lib.lib()
fake = ctypes.c_void_p(256)   # never dereferenced: the size check comes first
cases = [(65536, 65536, 2**31 - 1), (46341, 1, 1), (1, 46341, 1), (1448, 1448, 2),
         (1, 1, 2**31 - 1), (2048, 1024, 1), (3, 5, 2**21 // 15 + 1)]
print([L.pllgpu_dct2d_batch_noalloc(0, a, b, h, fake, fake, None) for a, b, h in cases])
"""


def test_noalloc_size_check_rejects_overflowing_requests_without_a_gpu():
    """Requests whose scratch size overflows a 64-bit product or exceeds the
    fixed array come back PLLGPU_EINVAL before any device work: run where no
    GPU is visible, a call that got past the check would fail in
    cudaGetDevice (PLLGPU_ECUDA) instead."""
    import subprocess
    import sys

    from pllcart3d_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libpllgpu.so not built")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", _NOALLOC_OVERFLOW, ROOT], env=env, capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip().splitlines()[-1] == "[5, 5, 5, 5, 5, 5, 5]", out.stdout
