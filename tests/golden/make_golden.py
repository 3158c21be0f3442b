"""Regenerate the golden vectors in this folder from the reference itself.

Runs the reference's own pllcart3d.c step routines, compiled by
oracle/Makefile (``make -C oracle ref``; needs the reference sources), on
seeded synthetic fingering cases and stores the FP64 state they produce:

* ``ref_16x8x8_s3.npz``   - every state field after 3 steps of a 16x8x8 case;
* ``ref_12x6x10_s4.npz``  - an uneven grid (ny != nz) with body forces Fx, Fy;
* ``ref_64x32x32_s200_summary.json`` - per-field max-norm, sum and a fixed
  sample of entries after the full 200-step 64x32x32 run.

Usage: python tests/golden/make_golden.py
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.pyref import FIELDS, RefRun  # noqa: E402
from pllcart3d_b200.ic import workload_fields  # noqa: E402
from pllcart3d_b200.params import workload  # noqa: E402

SAMPLE_SEED = 7


def small_case(name, steps, **kw):
    wl = workload(name)
    wl.params = wl.params.replace(**kw)
    ic = workload_fields(wl)
    r = RefRun(wl.params, ic)
    r.steps(steps)
    out = {f: r.get(f) for f in FIELDS}
    for k, v in ic.items():
        out["ic_" + k] = v
    out["dt"] = np.array([r.dt])
    return out


def summary(state):
    rng = np.random.default_rng(SAMPLE_SEED)
    res = {}
    for f, a in state.items():
        idx = [tuple(int(rng.integers(0, s)) for s in a.shape) for _ in range(16)]
        res[f] = {"maxabs": float(np.abs(a).max()), "sum": float(a.sum()),
                  "sample_idx": idx, "sample": [float(a[i]) for i in idx]}
    return res


def main():
    np.savez_compressed(os.path.join(HERE, "ref_16x8x8_s3.npz"),
                        **small_case("fingering-16x8x8", 3))
    np.savez_compressed(os.path.join(HERE, "ref_12x6x10_s4.npz"),
                        **small_case("fingering-12x6x10", 4, Fx=2.0, Fy=-1.5))
    wl = workload("fingering-64x32x32")
    r = RefRun(wl.params, workload_fields(wl))
    r.steps(wl.steps)
    st = {f: r.get(f) for f in ("c_new", "u_new", "v_new", "w_new", "phi",
                                "u_pg", "v_pg", "w_pg")}
    with open(os.path.join(HERE, "ref_64x32x32_s200_summary.json"), "w") as f:
        json.dump({"steps": wl.steps, "last_dt": r.dt, "fields": summary(st)},
                  f, indent=1)


if __name__ == "__main__":
    main()
