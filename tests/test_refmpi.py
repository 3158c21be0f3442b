"""The reference's multi-rank CPU path (oracle/refmpi.py over the
shared-memory MPI stand-in oracle/shim/shmmpi.c) against its single-rank
path: one rank over the stand-in is the single-rank reference bit for bit,
and the x-slab runs on 2 and 4 ranks stay within the reference's own
rank-count dependence (its ENO-2 closure reads scratch that the previous
sweep left, which depends on the slab width; pllcart3d.c:1545-1546)."""

import numpy as np
import pytest

import oracle.pyref as pyref
from oracle import refmpi
from pllcart3d_b200.ic import workload_fields
from pllcart3d_b200.params import workload

pytestmark = pytest.mark.skipif(not (refmpi.available() and pyref.ref_available()),
                                reason="reference libraries not built")


def test_one_rank_over_the_stand_in_is_the_single_rank_reference():
    wl = workload("fingering-32x16x16")
    ic = workload_fields(wl)
    r = refmpi.run(wl.params, ic, 1, 0, 4, want_c=True)
    a = pyref.RefRun(wl.params, ic)
    a.set_fast_dct(True)
    a.steps(4)
    assert np.array_equal(r["c_new"], a.get("c_new"))


@pytest.mark.parametrize("ranks", [2, 4])
def test_slab_decomposition_tracks_one_rank(ranks):
    wl = workload("fingering-32x16x16")
    ic = workload_fields(wl)
    one = refmpi.run(wl.params, ic, 1, 0, 4, want_c=True)["c_new"]
    many = refmpi.run(wl.params, ic, ranks, 1, 3, want_c=True)
    assert many["seconds"] > 0
    assert float(np.abs(many["c_new"] - one).max()) <= 1e-6
