"""Ensembles (one graph launch per step for all members) and the launch-shape
autotuner: every member must equal its own single run bit for bit, and a
tuned run the untuned run of the same number of steps."""

import numpy as np
import pytest

from pllcart3d_b200.ic import workload_fields
from pllcart3d_b200.params import Workload, workload

pytestmark = pytest.mark.gpu

FIELDS = ("c_new", "u_new", "v_new", "w_new", "phi", "u_pg", "c_hn")


def _members(specs):
    base = workload("fingering-64x32x32")
    out = []
    for n, (grid, R, Pe, Re) in enumerate(specs):
        p = base.params.replace(Nx_cell_global=grid[0], Ny_cell_global=grid[1], Nz_cell_global=grid[2],
                                Vratio=-R, Pe=Pe, Re=Re)
        out.append(Workload(f"m{n}", p, modes=8, amplitude=0.01, seed=1000 + n))
    return out


def _single(w, precision, steps, tuning=None):
    from pllcart3d_b200.solver import Solver

    s = Solver(w.params, precision=precision)
    s.load_ic(workload_fields(w))
    if tuning is not None:
        s.set_tuning(*tuning)
    s.step(steps)
    return s


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_members_equal_single_runs(precision):
    from pllcart3d_b200.ensemble import Ensemble

    specs = [((16, 8, 8), 2.0, 1000.0, 100.0), ((24, 12, 12), 0.5, 700.0, 400.0),
             ((32, 16, 16), 2.9, 3000.0, 900.0), ((16, 16, 16), 1.2, 500.0, 250.0)]
    if precision == "mixed":
        specs.append(((8, 128, 128), 1.5, 2000.0, 500.0))   # tcgen05 DCT passes
    wls = _members(specs)
    ens = Ensemble(wls, precision=precision)
    ens.load_ics()
    ens.step(3)
    ens.step(4)
    assert ens.launches_per_step > 0
    for m, w in zip(ens.members, wls):
        s = _single(w, precision, 7)
        for f in FIELDS:
            assert np.array_equal(m.get(f), s.get(f)), (w.name, f)
        assert m.tval == s.tval
    ens.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed64", "mixed"])
def test_batched_classes_equal_single_runs(precision):
    """Members sharing a grid form a class that issues one launch per stage
    (a kernel body over all of the class's members): every member still
    equals its own single run bit for bit, and the batched graph issues
    fewer launches than one branch per member."""
    from pllcart3d_b200.ensemble import Ensemble

    specs = [((16, 8, 8), 2.0, 1000.0, 100.0), ((24, 12, 12), 0.5, 700.0, 400.0),
             ((16, 8, 8), 0.7, 2500.0, 800.0), ((24, 12, 12), 2.6, 900.0, 150.0),
             ((16, 8, 8), 1.4, 600.0, 300.0), ((32, 16, 16), 2.9, 3000.0, 900.0)]
    classes = 3
    if precision == "mixed":
        # a class whose DCT passes (tcgen05, tensor-map arguments) replay
        # per member inside the batched branch
        specs += [((8, 128, 128), 1.5, 2000.0, 500.0), ((8, 128, 128), 0.4, 1200.0, 200.0)]
        classes = 4
    wls = _members(specs)
    ens = Ensemble(wls, precision=precision)
    ens.load_ics()
    ens.step(3)
    assert ens.classes == classes
    batched = ens.launches_per_step
    ens.step(4)
    for m, w in zip(ens.members, wls):
        s = _single(w, precision, 7)
        for f in FIELDS:
            assert np.array_equal(m.get(f), s.get(f)), (w.name, f)
        assert m.tval == s.tval
    # one branch per member: same results, more launches
    assert ens.set_batching(False)
    ens.step(2)
    assert ens.classes == len(wls)
    assert ens.launches_per_step > batched
    for m, w in zip(ens.members, wls):
        s = _single(w, precision, 9)
        assert np.array_equal(m.get("c_new"), s.get("c_new")), w.name
    # classes split into groups of at most 2 members, one branch each
    assert ens.set_batching(2) == 0
    ens.step(2)
    assert ens.classes == classes + 1   # the 3-member class makes 2 groups
    assert batched < ens.launches_per_step
    for m, w in zip(ens.members, wls):
        s = _single(w, precision, 11)
        for f in FIELDS:
            assert np.array_equal(m.get(f), s.get(f)), (w.name, f)
    ens.close()


def test_autotune_changes_timing_only():
    from pllcart3d_b200.solver import Solver

    w = workload("fingering-32x16x16")
    a = Solver(w.params)
    a.load_ic(workload_fields(w))
    done = a.autotune(1)
    assert done == 4 * 3 * 2
    a.step(2)
    b = _single(w, "fp64", done + 2)
    for f in FIELDS:
        assert np.array_equal(a.get(f), b.get(f)), f
    # every variant by hand
    for ve in range(4):
        for vl in range(3):
            c = _single(w, "fp64", 3, tuning=(ve, vl))
            d = _single(w, "fp64", 3)
            assert np.array_equal(c.get("u_new"), d.get("u_new")), (ve, vl)


def test_ensemble_autotune_and_restarted_member(tmp_path):
    from pllcart3d_b200.ensemble import Ensemble
    from pllcart3d_b200.solver import Solver

    wls = _members([((16, 8, 8), 2.0, 1000.0, 100.0), ((16, 16, 16), 1.0, 800.0, 300.0)])
    ens = Ensemble(wls, precision="fp64")
    ens.load_ics()
    done = ens.autotune(1)
    ens.step(2)
    for m, w in zip(ens.members, wls):
        s = _single(w, "fp64", done + 2)
        assert np.array_equal(m.get("c_new"), s.get("c_new"))
    # member 0 restarts from its own restart files and the ensemble steps on
    m0 = ens.members[0]
    m0.write_restart(done + 2, 0, m0.tval, 0.0, 0.0, 0.0, str(tmp_path))
    m0.read_restart(str(tmp_path))
    ens.step(3)
    s = _single(wls[1], "fp64", done + 5)
    assert np.array_equal(ens.members[1].get("u_new"), s.get("u_new"))
    ens.close()
