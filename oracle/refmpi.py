"""The reference's own multi-rank CPU step, timed on the host cores.

Runs pllcart3d.c's time step on its x-slab decomposition (grid_setup,
pllcart3d.c:357-378; halo exchanges L2230-2696; pll_tridiag.c's pipelined x
solves) as `ranks` processes over the project's shared-memory MPI stand-in
(oracle/shim/shmmpi.c), from the same seeded initial fields the GPU runs.
Measurement infrastructure only (the reference arm and CPU baseline of
bench.py, and tests): the GPU library never loads it.

    python -m oracle.refmpi --workload fingering-512x256x256 --ranks 16 --warmup 1 --steps 2
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
MPI_LIB = os.path.join(HERE, "_ref", "libpllref_mpi.so")


def available() -> bool:
    return os.path.exists(MPI_LIB)


def max_ranks(nx: int) -> int:
    """Ranks the slab decomposition allows: every slab needs at least the 3
    planes its neighbours' halos read."""
    return max(1, nx // 3)


def run(params, ic, ranks: int, warm: int, steps: int, want_c: bool = False, budget_s: float = 0.0) -> dict:
    """`warm` untimed steps, then up to `steps` timed ones (fewer once
    `budget_s` seconds have passed; 0 = no limit)."""
    if not available():
        raise FileNotFoundError(MPI_LIB)
    lib = ctypes.CDLL(MPI_LIB, mode=os.RTLD_LOCAL)
    P = ctypes.POINTER(ctypes.c_double)
    lib.pllref_mpi_run.argtypes = [ctypes.c_int, ctypes.c_char_p, P, P, P, P, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, P, ctypes.c_long, ctypes.c_int, P]
    arrs = [np.ascontiguousarray(ic[k], dtype=np.float64) for k in "cuvw"]
    out = np.zeros(4)
    c_out = np.zeros(params.shape) if want_c else None
    with tempfile.TemporaryDirectory(prefix="pllrefmpi_") as d:
        params.write(d)
        rc = lib.pllref_mpi_run(int(ranks), d.encode(), *[a.ctypes.data_as(P) for a in arrs], int(warm),
                                int(steps), float(budget_s), out.ctypes.data_as(P), int(np.prod(params.shape)),
                                int(params.shape[0]), c_out.ctypes.data_as(P) if want_c else None)
    if rc != 0:
        raise RuntimeError(f"reference MPI run failed (rc {rc})")
    done = int(out[3])
    res = {"ranks": ranks, "steps": done, "warmup": warm, "seconds": float(out[0]),
           "warmup_seconds": float(out[1]), "setup_seconds": float(out[2]),
           "cell_steps_per_s": params.cells * done / float(out[0]) if out[0] > 0 else None}
    if want_c:
        res["c_new"] = c_out
    return res


def main(argv=None) -> int:
    sys.path.insert(0, ROOT)
    from pllcart3d_b200.ic import workload_fields
    from pllcart3d_b200.params import workload

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="fingering-512x256x256")
    ap.add_argument("--ranks", type=int, default=0, help="0: every host core the slabs allow")
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--budget", type=float, default=0.0, help="seconds after which timed steps stop")
    args = ap.parse_args(argv)
    wl = workload(args.workload)
    ranks = args.ranks or min(os.cpu_count() or 1, max_ranks(wl.params.nx))
    res = run(wl.params, workload_fields(wl), ranks, args.warmup, args.steps, budget_s=args.budget)
    res.update({"workload": wl.name, "cells": wl.params.cells, "host_cores": os.cpu_count()})
    print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
