"""Accuracy of one form of the step against another (default: the precision
form against the plain FP64 step).

    python -m pllcart3d_b200.validate [--workload NAME] [--steps N] [--every K]
                                      [--test FORM] [--ref FORM]

FORM: fp64 (the FP64 form), fp64-exact (the reference's operation order,
sequential-order DCT), mixed64 (FP64 state, FP32 WENO5 weights), mixed (tcgen05
split-TF32 DCT where the shape allows), mixed-mma (mma.sync split-TF32 DCT),
mixed-seq (sequential FP32 DCT).  Both runs start from the same seeded
initial condition and advance in lockstep; every K steps (or at the steps
listed by --at) the relative max-norm error of each field (velocity
components against the velocity vector's max-norm) and the FP64 diagnostics
of both (mass, divergence norms, mixing length) are printed, one JSON line
per checkpoint.

--perturb REL multiplies the test run's initial c (the whole padded box) by
(1 + REL s), s a seeded random field of +-1: with --test fp64 --ref fp64 and
REL = 6e-8 (one FP32 rounding) it measures how far the flow itself carries a
single rounding-sized perturbation, the sensitivity against which a form
with FP32 arithmetic is judged.
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
VECTORS = {"u_new": ("u_new", "v_new", "w_new"), "v_new": ("u_new", "v_new", "w_new"),
           "w_new": ("u_new", "v_new", "w_new"), "u_pg": ("u_pg", "v_pg", "w_pg"),
           "v_pg": ("u_pg", "v_pg", "w_pg"), "w_pg": ("u_pg", "v_pg", "w_pg")}
FORMS = {"fp64": dict(precision="fp64"), "fp64-exact": dict(precision="fp64", exact_dct=True),
         "mixed": dict(precision="mixed"), "mixed-mma": dict(precision="mixed", dct_kernel="mma_sync"),
         "mixed64": dict(precision="mixed64"),
         "mixed-seq": dict(precision="mixed", exact_dct=True)}


def rel(test, ref, f) -> float:
    den = max(float(np.abs(ref.get(c)).max()) for c in VECTORS.get(f, (f,)))
    num = float(np.abs(test.get(f) - ref.get(f)).max())
    return num / den if den > 0 else num


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="fingering-512x256x256")
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--every", type=int, default=250)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--test", default="mixed", choices=sorted(FORMS))
    ap.add_argument("--ref", default="fp64", choices=sorted(FORMS))
    ap.add_argument("--at", default=None, help="comma-separated checkpoint steps (instead of --every)")
    ap.add_argument("--perturb", type=float, default=0.0, help="relative +-perturbation of the test run's c")
    ap.add_argument("--perturb-seed", type=int, default=20240601)
    ap.add_argument("--out", default=None, help="also append the JSON lines to this file")
    args = ap.parse_args(argv)
    wl = workload(args.workload)
    ic = workload_fields(wl)
    ic_test = ic
    if args.perturb:
        sgn = np.random.default_rng(args.perturb_seed).integers(0, 2, ic["c"].shape) * 2.0 - 1.0
        ic_test = dict(ic)
        ic_test["c"] = ic["c"] * (1.0 + args.perturb * sgn)
    ref = Solver(wl.params, device=args.device, **FORMS[args.ref])
    mix = Solver(wl.params, device=args.device, **FORMS[args.test])
    marks = sorted(int(t) for t in args.at.split(",")) if args.at else None
    ref.load_ic(ic)
    mix.load_ic(ic_test)
    done = 0
    t_ref = t_mix = 0.0
    last = marks[-1] if marks else args.steps
    while done < last:
        n = (next(m for m in marks if m > done) - done) if marks else min(args.every, args.steps - done)
        t0 = time.perf_counter()
        ref.step(n)
        t1 = time.perf_counter()
        mix.step(n)
        t2 = time.perf_counter()
        t_ref += t1 - t0
        t_mix += t2 - t1
        done += n
        errs = {f: rel(mix, ref, f) for f in FIELDS}
        line = {"workload": wl.name, "test": args.test, "ref": args.ref, "steps": done,
                "rel_maxnorm": errs, "diag_ref": ref.diagnostics(), "diag_test": mix.diagnostics(),
                "dt_ref": ref.dt, "dt_test": mix.dt, "tval_ref": ref.tval, "tval_test": mix.tval,
                "wall_s_ref": t_ref, "wall_s_test": t_mix, "perturb": args.perturb}
        print(json.dumps(line), flush=True)
        if args.out:
            with open(args.out, "a") as f:
                f.write(json.dumps(line) + "\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
