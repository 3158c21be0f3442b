"""The no-allocation DCT entry point against the allocating one.

pllgpu_dct2d_batch_noalloc exists for callers that cannot allocate device
memory (their pool allocator owns the device, or the device synchronisation
of cudaMalloc/cudaFree is not acceptable to them): it uses the caller's
device buffers for input and output and a fixed scratch array inside the
library for everything else.  This file is collected last on purpose, so a
run that stops at the first failure has run every other test first.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # the DCT tolerance of the other GPU tests


def _noalloc(L, kind, x_dev, out_dev, stream):
    n0, n1 = x_dev.shape[-2:]
    howmany = x_dev.numel() // (n0 * n1)
    return L.pllgpu_dct2d_batch_noalloc(kind, n0, n1, howmany, ctypes.c_void_p(x_dev.data_ptr()),
                                        ctypes.c_void_p(out_dev.data_ptr()), ctypes.c_void_p(stream))


def test_noalloc_dct_matches_allocating_entry_point_twice():
    import torch

    from pllcart3d_b200 import _lib
    from pllcart3d_b200.solver import dct2d_batch

    L = _lib.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(11)
    cases = [(0, (6, 24, 40)), (1, (5, 32, 16))]   # two calls in a row
    for kind, shape in cases:
        x = rng.standard_normal(shape)
        want = dct2d_batch(kind, x)
        x_dev = torch.from_numpy(x).cuda()
        out_dev = torch.full(shape, float("nan"), dtype=torch.float64, device="cuda")
        assert _noalloc(L, kind, x_dev, out_dev, stream) == 0
        torch.cuda.synchronize()
        got = out_dev.cpu().numpy()
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err <= REL_TOL, (kind, shape, err)


def test_noalloc_dct_rejects_sizes_beyond_its_scratch():
    import torch

    from pllcart3d_b200 import _lib

    L = _lib.lib()
    torch.cuda.set_device(0)
    n0 = n1 = 512
    howmany = (1 << 21) // (n0 * n1) + 1
    x = torch.zeros((howmany, n0, n1), dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    assert _noalloc(L, 0, x, y, torch.cuda.current_stream().cuda_stream) == 5  # PLLGPU_EINVAL
