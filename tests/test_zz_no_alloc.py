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


def _check(L, kind, x, stream):
    import torch

    from pllcart3d_b200.solver import dct2d_batch

    want = dct2d_batch(kind, x)
    x_dev = torch.from_numpy(x).cuda()
    out_dev = torch.full(x.shape, float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert _noalloc(L, kind, x_dev, out_dev, stream) == 0
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    got = out_dev.cpu().numpy()
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err <= REL_TOL, (kind, x.shape, err)
    return free0, free1


def test_noalloc_dct_matches_allocating_entry_point_twice():
    import torch

    from pllcart3d_b200 import _lib

    L = _lib.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(11)
    # two calls in a row; the second finds the first's matrices and
    # intermediate in the shared scratch and must not depend on them.  The
    # device's free memory does not move across the second call (the first
    # call on a device only looks up the scratch array's address).
    _check(L, 0, rng.standard_normal((6, 24, 40)), stream)
    free0, free1 = _check(L, 1, rng.standard_normal((5, 32, 16)), stream)
    assert free1 == free0, (free0, free1)


def test_noalloc_dct_runs_batches_beyond_one_grid_dimension():
    """70000 small arrays fit the scratch; the call launches them in chunks
    of at most 65535 (the grid's z limit)."""
    import torch

    from pllcart3d_b200 import _lib

    L = _lib.lib()
    torch.cuda.set_device(0)
    rng = np.random.default_rng(12)
    _check(L, 0, rng.standard_normal((70000, 2, 2)), torch.cuda.current_stream().cuda_stream)


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
