"""Accuracy of the precision form against the plain FP64 step.

    python -m pllcart3d_b200.validate [--workload NAME] [--steps N] [--every K]

Both forms start from the same seeded initial condition and advance in
lockstep; every K steps the relative max-norm error of each field of the
precision form (max|mixed - fp64| / max|fp64| over the padded box) and the
FP64 diagnostics of both (mass, divergence norms, mixing length) are
printed, one JSON line per checkpoint.
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .ic import workload_fields
from .params import workload
from .solver import Solver

FIELDS = ("c_new", "u_new", "v_new", "w_new", "phi", "u_pg", "v_pg", "w_pg")


def rel(a: np.ndarray, b: np.ndarray) -> float:
    den = float(np.abs(b).max())
    return float(np.abs(a - b).max()) / den if den > 0 else float(np.abs(a - b).max())


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="fingering-512x256x256")
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--every", type=int, default=250)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    wl = workload(args.workload)
    ic = workload_fields(wl)
    ref = Solver(wl.params, device=args.device, precision="fp64")
    mix = Solver(wl.params, device=args.device, precision="mixed")
    ref.load_ic(ic)
    mix.load_ic(ic)
    done = 0
    t_ref = t_mix = 0.0
    while done < args.steps:
        n = min(args.every, args.steps - done)
        t0 = time.perf_counter()
        ref.step(n)
        t1 = time.perf_counter()
        mix.step(n)
        t2 = time.perf_counter()
        t_ref += t1 - t0
        t_mix += t2 - t1
        done += n
        errs = {f: rel(mix.get(f), ref.get(f)) for f in FIELDS}
        line = {"workload": wl.name, "steps": done, "rel_maxnorm": errs,
                "diag_fp64": ref.diagnostics(), "diag_mixed": mix.diagnostics(),
                "dt_fp64": ref.dt, "dt_mixed": mix.dt, "tval_fp64": ref.tval,
                "tval_mixed": mix.tval, "wall_s_fp64": t_ref, "wall_s_mixed": t_mix}
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
