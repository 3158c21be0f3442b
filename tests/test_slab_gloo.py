"""The x-slab decomposition's collectives (pllcart3d_b200/slab.py) on CPU
with 2 and 4 gloo ranks: the partitioned x-tridiagonal solve against one
Thomas sweep over the whole systems, the halo exchange against the
neighbours' planes, the fused scalar reduction, and the reference's slab
sizes."""

import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _systems(N, n, seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1.0, -0.1, (N, n))
    c = rng.uniform(-1.0, -0.1, (N, n))
    b = 2.5 + rng.uniform(0.0, 1.0, (N, n))
    r = rng.standard_normal((N, n))
    return a, b, c, r


def _thomas(a, b, c, r):
    N, n = r.shape
    cp = np.zeros((N, n))
    rp = np.zeros((N, n))
    cp[:, 0] = c[:, 0] / b[:, 0]
    rp[:, 0] = r[:, 0] / b[:, 0]
    for i in range(1, n):
        d = b[:, i] - a[:, i] * cp[:, i - 1]
        cp[:, i] = c[:, i] / d
        rp[:, i] = (r[:, i] - a[:, i] * rp[:, i - 1]) / d
    x = np.zeros((N, n))
    x[:, -1] = rp[:, -1]
    for i in range(n - 2, -1, -1):
        x[:, i] = rp[:, i] - cp[:, i] * x[:, i + 1]
    return x


def _worker(rank, ws, port, q, n):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    from pllcart3d_b200 import slab

    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    res = {}
    # partitioned solve of the same systems every rank generated
    a, b, c, r = _systems(37, n, 5)
    off, m = slab.slab_ranges(n, ws)[rank]
    t = [torch.from_numpy(np.ascontiguousarray(z[:, off:off + m])) for z in (a, b, c, r)]
    res["x"] = slab.partitioned_tridiag(*t).numpy()
    res["range"] = (off, m)
    # halo exchange (every rank takes the same branch: slabs of at least 3
    # planes): plane p of the global field holds the value p everywhere
    w = 3
    res["halo"] = None
    if min(k for _, k in slab.slab_ranges(n, ws)) >= w:
        f = torch.full((w + m + w, 4, 5), -1.0, dtype=torch.float64)
        for i in range(m):
            f[w + i] = off + i
        slab.halo_exchange(f, w)
        res["halo"] = (f[:w, 0, 0].tolist(), f[w + m:, 0, 0].tolist())
    # fused scalars
    res["scal"] = slab.reduce_scalars(1.0 + rank, qin=2.5 if rank == 0 else None,
                                      qout=3.5 if rank == ws - 1 else None,
                                      vbulk=-0.75 if rank == ws - 1 else None)
    q.put((rank, res))
    dist.destroy_process_group()


# (4, 6): slabs of 2, 2, 1 and 1 rows (one-row blocks in the solve)
@pytest.mark.parametrize("ws,n", [(2, 23), (4, 30), (4, 6)])
def test_slab_collectives(ws, n):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q, n)) for r in range(ws)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b, c, r = _systems(37, n, 5)
    want = _thomas(a, b, c, r)
    got = np.concatenate([out[k]["x"] for k in range(ws)], axis=1)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    for k in range(ws):
        off, m = out[k]["range"]
        if out[k]["halo"] is not None:
            lo, hi = out[k]["halo"]
            assert lo == ([-1.0] * 3 if k == 0 else [float(off - 3 + i) for i in range(3)])
            assert hi == ([-1.0] * 3 if k == ws - 1 else [float(off + m + i) for i in range(3)])
        assert out[k]["scal"] == (float(ws), 2.5, 3.5, -0.75)


def test_slab_ranges_follow_grid_setup():
    sys.path.insert(0, ROOT)
    from pllcart3d_b200.slab import slab_ranges

    # (nx + size - r - 1) // size cells per rank, in rank order
    assert slab_ranges(10, 4) == [(0, 3), (3, 3), (6, 2), (8, 2)]
    assert slab_ranges(512, 16) == [(32 * r, 32) for r in range(16)]
    assert sum(n for _, n in slab_ranges(257, 7)) == 257
