"""Ensembles of independent fingering runs advanced together on one GPU.

``Ensemble`` wraps the ``pllgpu_ensemble_*`` C ABI: every member is an
ordinary context (``Ensemble.members[i]`` is a :class:`Solver` view of it)
and one CUDA graph launch advances every member by one step.  Members of one
grid form a class that issues one launch per stage for all of its members
(``set_batching(False)``: one graph branch per member instead).
``random_members`` draws the members of the
ensemble workload: grids from {32^3, 64x32x32, 64^3, 128x64x64}, R ~ U[0,3],
Pe log-uniform in [500, 5000], Re ~ U[100, 1000], the 64x32x32 workload's
interface recipe with a per-member seed.

    python -m pllcart3d_b200.ensemble [--members 64] [--steps 500]
                                      [--precision mixed] [--snapshots DIR]

prints one JSON line: aggregate cell-steps/s of the ensemble graph against
the same members run one after another (each alone, graph-stepped), with
every member's result checked equal between the two, and (--branches) the
rate of the graph with one branch per member.  With --snapshots,
every 8th step's (c, u, v, w) interior of every member goes to DIR as
``member%03d.npz`` (the surrogate's training data).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import time

import numpy as np

from . import _lib
from .ic import workload_fields
from .params import Params, Workload, workload
from .solver import Solver

GRIDS = ((32, 32, 32), (64, 32, 32), (64, 64, 64), (128, 64, 64))


def random_members(n: int, seed: int = 1234) -> list:
    """The ensemble workload's members (deterministic in `seed`)."""
    rng = np.random.default_rng(seed)
    base = workload("fingering-64x32x32")
    out = []
    for m in range(n):
        nx, ny, nz = GRIDS[int(rng.integers(len(GRIDS)))]
        R = float(rng.uniform(0.0, 3.0))
        Pe = float(math.exp(rng.uniform(math.log(500.0), math.log(5000.0))))
        Re = float(rng.uniform(100.0, 1000.0))
        p = base.params.replace(Nx_cell_global=nx, Ny_cell_global=ny, Nz_cell_global=nz,
                                Vratio=-R, Pe=Pe, Re=Re)
        out.append(Workload(f"member{m:03d}-{nx}x{ny}x{nz}", p, modes=base.modes,
                            amplitude=base.amplitude, steps=500, seed=base.seed + 7919 * (m + 1)))
    return out


class Ensemble:
    def __init__(self, workloads, precision: str = "mixed", device: int = 0):
        self.workloads = list(workloads)
        self.precision = precision
        self._L = _lib.lib()
        arr = (_lib.Params * len(self.workloads))()
        for i, w in enumerate(self.workloads):
            arr[i] = Solver.c_params(w.params, precision=precision)
        self._h = self._L.pllgpu_ensemble_create(len(self.workloads), arr, int(device))
        if not self._h:
            raise _lib.PllGpuError(2, "pllgpu_ensemble_create")
        self.members = [Solver.view(self._L.pllgpu_ensemble_member(self._h, i), w.params, precision)
                        for i, w in enumerate(self.workloads)]

    def close(self) -> None:
        if getattr(self, "_h", None):
            for m in self.members:
                m.close()
            self._L.pllgpu_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code: int, what: str) -> None:
        if code != 0:
            raise _lib.PllGpuError(code, what)

    def load_ics(self) -> None:
        for m, w in zip(self.members, self.workloads):
            ic = workload_fields(w)
            for k in "cuvw":
                m.set(f"{k}_new", ic[k])
        self._check(self._L.pllgpu_ensemble_start(self._h), "ensemble_start")

    def step(self, n: int = 1) -> None:
        self._check(self._L.pllgpu_ensemble_steps(self._h, int(n)), "ensemble_steps")

    def autotune(self, trial_steps: int = 1) -> int:
        done = ctypes.c_int()
        self._check(self._L.pllgpu_ensemble_autotune(self._h, int(trial_steps), ctypes.byref(done)),
                    "ensemble_autotune")
        return done.value

    @property
    def launches_per_step(self) -> int:
        return self._L.pllgpu_ensemble_launches_per_step(self._h)

    @property
    def classes(self) -> int:
        """Branches (classes of members with the same launches, or groups of
        a class) of the graphs last built."""
        return self._L.pllgpu_ensemble_classes(self._h)

    def set_batching(self, mode) -> int:
        """1 / True (the default): one launch per stage and class; k >= 2:
        classes split into groups of at most k members; 0 / False: every
        member's own launches as its own branch.  Returns the previous mode."""
        old = self._L.pllgpu_ensemble_set_batching(self._h, int(mode))
        if old < 0:
            raise _lib.PllGpuError(-old, "ensemble_set_batching")
        return old

    def cells(self) -> int:
        return sum(w.params.nx * w.params.ny * w.params.nz for w in self.workloads)


def interior(p: Params, a: np.ndarray) -> np.ndarray:
    return a[3:p.nx + 3, 1:p.ny + 1, 1:p.nz + 1]


def snapshot_state(s: Solver) -> np.ndarray:
    """(4, nx, ny, nz) float32: c and the cell-centred u, v, w."""
    p = s.params
    c, u, v, w = (s.get(f"{q}_new") for q in "cuvw")
    I, J, K = slice(3, p.nx + 3), slice(1, p.ny + 1), slice(1, p.nz + 1)
    uc = 0.5 * (u[I, J, K] + u[4:p.nx + 4, J, K])
    vc = 0.5 * (v[I, J, K] + v[I, 2:p.ny + 2, K])
    wc = 0.5 * (w[I, J, K] + w[I, J, 2:p.nz + 2])
    return np.stack([c[I, J, K], uc, vc, wc]).astype(np.float32)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed64", "mixed"])
    ap.add_argument("--out", default=None, help="also write the report JSON to this file")
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--snapshots", default=None)
    ap.add_argument("--every", type=int, default=8)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--branches", type=int, default=100,
                    help="also time this many steps of the graph with one branch per member (0: skip)")
    ap.add_argument("--group", type=int, default=1,
                    help="members per batched launch at most (1: whole classes)")
    args = ap.parse_args(argv)
    import torch

    wls = random_members(args.members, args.seed)
    ens = Ensemble(wls, precision=args.precision)
    ens.load_ics()
    tuned_steps = 0 if args.no_tune else ens.autotune(1)
    done = tuned_steps
    branch = None
    if args.branches > 0:
        # every member's own launches, one graph branch per member
        ens.set_batching(False)
        ens.step(2)   # warm-up, graph capture
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ens.step(args.branches)
        torch.cuda.synchronize()
        branch = {"cell_steps_per_s": ens.cells() * args.branches / (time.perf_counter() - t0),
                  "launches_per_graph_step": ens.launches_per_step, "steps": args.branches}
        done += 2 + args.branches
    ens.set_batching(args.group)
    ens.step(2)   # warm-up, graph capture
    torch.cuda.synchronize()
    done += 2
    snaps = {i: [] for i in range(len(wls))} if args.snapshots else None
    t0 = time.perf_counter()
    timed = 0
    while done < args.steps:
        n = min(args.every, args.steps - done) if snaps is not None else args.steps - done
        ens.step(n)
        done += n
        timed += n
        if snaps is not None:
            t_pause = time.perf_counter()
            for i, m in enumerate(ens.members):
                snaps[i].append(snapshot_state(m))
            t0 += time.perf_counter() - t_pause   # snapshot copies are not step time
    t_ens = time.perf_counter() - t0
    ens_cells = ens.cells() * timed / t_ens

    # the same members one after another, each alone
    t_seq = 0.0
    mismatches = 0
    for i, w in enumerate(wls):
        s = Solver(w.params, precision=args.precision)
        s.load_ic(workload_fields(w))
        e_var, l_var = ens.members[i].tuning()
        s.set_tuning(e_var, l_var)
        s.step(done - timed)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        s.step(timed)
        t_seq += time.perf_counter() - t1
        for q in "cuvw":
            if not np.array_equal(s.get(f"{q}_new"), ens.members[i].get(f"{q}_new")):
                mismatches += 1
        s.close()
    seq_cells = ens.cells() * timed / t_seq
    if snaps is not None:
        os.makedirs(args.snapshots, exist_ok=True)
        for i, w in enumerate(wls):
            p = w.params
            np.savez(os.path.join(args.snapshots, f"member{i:03d}.npz"), states=np.stack(snaps[i]),
                     R=-p.Vratio, Pe=p.Pe, Re=p.Re, every=args.every)
    rep = {
        "workload": f"ensemble of {len(wls)} runs",
        "precision": args.precision, "steps": done, "timed_steps": timed,
        "cells": ens.cells(), "ensemble_cell_steps_per_s": ens_cells,
        "sequential_cell_steps_per_s": seq_cells, "speedup": ens_cells / seq_cells,
        "launches_per_graph_step": ens.launches_per_step, "branches": ens.classes, "group": args.group,
        "one_branch_per_member": branch, "autotune_steps": tuned_steps,
        "members_equal_to_single_runs": mismatches == 0,
        "grids": [list(w.params.shape) for w in wls]}
    print(json.dumps(rep))
    if args.out:
        with open(args.out, "w") as f:
            json.dump(rep, f, indent=1)
    ens.close()
    return 0 if mismatches == 0 else 1


if __name__ == "__main__":
    raise SystemExit(main())
