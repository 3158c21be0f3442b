"""The CPU restatement (oracle/) against the reference itself.

Two pins: the committed golden vectors produced by the reference's own
pllcart3d.c (tests/golden/make_golden.py), and - where the reference was
compiled here (oracle/_ref) - an in-process bitwise comparison on cases the
golden files do not cover.
"""

import json
import os

import numpy as np
import pytest

from oracle.pyref import FIELDS, OracleRun, RefRun, ref_available
from pllcart3d_b200.ic import workload_fields
from pllcart3d_b200.params import workload

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _run_oracle(name, steps, **kw):
    wl = workload(name)
    wl.params = wl.params.replace(**kw)
    o = OracleRun(wl.params, workload_fields(wl))
    o.steps(steps)
    return o


@pytest.mark.parametrize("fname,name,steps,kw", [
    ("ref_16x8x8_s3.npz", "fingering-16x8x8", 3, {}),
    ("ref_12x6x10_s4.npz", "fingering-12x6x10", 4, {"Fx": 2.0, "Fy": -1.5}),
])
def test_oracle_matches_golden_bitwise(fname, name, steps, kw):
    g = np.load(os.path.join(GOLD, fname))
    wl = workload(name)
    wl.params = wl.params.replace(**kw)
    ic = workload_fields(wl)
    for k in "cuvw":
        assert np.array_equal(ic[k], g["ic_" + k]), "IC generator drifted"
    o = _run_oracle(name, steps, **kw)
    assert o.dt == float(g["dt"][0])
    for f in FIELDS:
        assert np.array_equal(o.get(f), g[f]), f


def test_oracle_matches_golden_summary_200_steps():
    with open(os.path.join(GOLD, "ref_64x32x32_s200_summary.json")) as f:
        gold = json.load(f)
    o = _run_oracle("fingering-64x32x32", gold["steps"])
    assert o.dt == gold["last_dt"]
    for name, s in gold["fields"].items():
        a = o.get(name)
        assert float(np.abs(a).max()) == s["maxabs"], name
        assert float(a.sum()) == s["sum"], name
        for idx, val in zip(s["sample_idx"], s["sample"]):
            assert float(a[tuple(idx)]) == val, (name, idx)


@pytest.mark.skipif(not ref_available(), reason="reference not compiled here")
@pytest.mark.parametrize("name,steps,kw", [
    ("fingering-20x6x9", 6, {}),
    ("fingering-18x9x7", 5, {"Nmvp": 1, "Vratio": 1.0, "Mum": 1.5}),
    ("fingering-16x8x8", 5, {"Re": 10.0, "Pe": 50.0, "CFLmax": 0.9}),
])
def test_oracle_matches_reference_inprocess(name, steps, kw):
    wl = workload(name)
    wl.params = wl.params.replace(**kw)
    ic = workload_fields(wl)
    r = RefRun(wl.params, ic)
    o = OracleRun(wl.params, ic)
    for _ in range(steps):
        r.steps(1)
        o.steps(1)
        assert r.dt == o.dt
    for f in FIELDS:
        assert np.array_equal(r.get(f), o.get(f)), f
