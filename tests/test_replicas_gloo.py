"""The N>1 path of bench.py (replicas, max-over-ranks timing) on CPU with
two gloo ranks."""

import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench

    t = bench.reduce_max(10.0 + 5.0 * rank, ws)   # per-rank step time, ms
    bench.barrier(ws)
    q.put((rank, t, bench.replica_value(1000, 4, ws, t)))
    dist.destroy_process_group()


def test_two_replicas_max_time_and_value():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]           # both see the slowest rank
    assert out[0][2] == 1000 * 4 * 2 / 0.015              # cells x steps x ranks / max time
