"""shift_conc (the spanwise wave perturbation, pllcart3d.c:3231-3344) on the
GPU against the compiled reference's own shift_conc on the same state, then
steps after it."""

import numpy as np
import pytest

from oracle import pyref
from pllcart3d_b200.ic import workload_fields
from pllcart3d_b200.params import workload

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not pyref.ref_available(), reason="reference library not built")]


@pytest.mark.parametrize("ampli,lamb,subharm", [(0.1, 0.5, 0), (0.03, 0.25, 1), (0.35, 1.0, 0)])
def test_shift_conc_matches_reference(ampli, lamb, subharm):
    from pllcart3d_b200.solver import Solver

    wl = workload("fingering-24x8x12")
    ic = workload_fields(wl)
    ref = pyref.RefRun(wl.params, ic)
    ref.steps(3)
    g = Solver(wl.params)
    g.load_ic(ic)
    g.step(3)
    ref.shift_conc(ampli, lamb, subharm)
    g.shift_conc(ampli, lamb, subharm)
    want = ref.get("c_old")
    got = g.get("c_old")
    assert np.abs(got - want).max() <= 1e-12, np.abs(got - want).max()
    # c_new keeps the unshifted field in both
    assert np.abs(g.get("c_new") - ref.get("c_new")).max() <= 1e-12
    ref.steps(4)
    g.step(4)
    for f in ("c_new", "u_new", "v_new", "w_new"):
        r = ref.get(f)
        assert np.abs(g.get(f) - r).max() <= 1e-10 * max(1.0, np.abs(r).max()), f
