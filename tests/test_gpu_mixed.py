"""The precision form (FP32 state and stencils, split-TF32 tensor-core DCT,
FP64 Poisson mode solve and reductions) against the FP64 GPU step from the
same seed, and the FP64 diagnostics against numpy."""

import numpy as np
import pytest

from pllcart3d_b200.ic import workload_fields
from pllcart3d_b200.params import workload
from tests.util import rel_maxnorm, rel_vector

pytestmark = pytest.mark.gpu


def _pair(name, steps):
    from pllcart3d_b200.solver import Solver

    wl = workload(name)
    ic = workload_fields(wl)
    a = Solver(wl.params, precision="fp64")
    b = Solver(wl.params, precision="mixed")
    a.load_ic(ic)
    b.load_ic(ic)
    a.step(steps)
    b.step(steps)
    return wl, a, b


def test_mixed_tracks_fp64_over_200_steps():
    wl, a, b = _pair("fingering-64x32x32", 200)
    errs = {f: rel_vector(b.get, a.get, f) for f in ("c_new", "u_new", "v_new", "w_new", "phi")}
    # FP32 state rounds at ~6e-8 per operation; the fingering flow amplifies
    # that noise, so after 200 steps c sits between 1e-5 and 2.5e-5 and the
    # velocity vector near 1e-5 of its max-norm (measured on B200; which
    # products are fused into one rounding moves c within that band: 0.9e-5
    # with single-cell arithmetic, 2.3e-5 with the paired FP32x2 explicit
    # operator, both at 1.3e-7 after one step)
    assert errs["c_new"] <= 5e-5, errs
    assert max(errs[f] for f in ("u_new", "v_new", "w_new")) <= 5e-5, errs
    assert errs["phi"] <= 1e-3, errs
    assert b.dt == pytest.approx(a.dt, rel=1e-5)


def test_mixed_routines_one_step():
    wl, a, b = _pair("fingering-32x16x16", 1)
    for f in ("c_new", "u_new", "u_pg"):
        assert rel_maxnorm(b.get(f), a.get(f)) <= 1e-5, f
    # phi is the potential of a near-cancelling divergence (FP32 velocity
    # differences lose ~3 digits); its FP32 error is ~3e-5 after one step
    assert rel_maxnorm(b.get("phi"), a.get("phi")) <= 1e-4


def test_paired_explicit_one_step():
    """The precision form's explicit operator computes cells (k, k+32) in
    pairs with packed FP32x2 instructions; on 64 z cells every thread's
    second cell is live.  One step agrees with the FP64 step to FP32 level."""
    wl, a, b = _pair("fingering-64x64x64", 1)
    assert b.status() == 0
    for f in ("c_new", "u_new", "v_new", "w_new"):
        assert rel_maxnorm(b.get(f), a.get(f)) <= 1e-4, f
    assert rel_maxnorm(b.get("c_new"), a.get("c_new")) <= 1e-6


@pytest.mark.parametrize("name", ["fingering-16x128x128", "fingering-8x256x256", "fingering-8x128x256"])
def test_tcgen05_dct_matches_mma_sync(name):
    """The tcgen05 split-TF32 DCT passes against the warp-level mma.sync
    split-TF32 passes, each measured against the FP64 step: both carry
    FP32-level products, so their errors agree to rounding."""
    from pllcart3d_b200.solver import Solver

    wl = workload(name)
    ic = workload_fields(wl)
    ref = Solver(wl.params, precision="fp64")
    tc = Solver(wl.params, precision="mixed")
    ms = Solver(wl.params, precision="mixed", dct_kernel="mma_sync")
    for s in (ref, tc, ms):
        s.load_ic(ic)
        s.step(1)
        assert s.status() == 0
    for f in ("phi", "u_new", "v_new", "w_new", "u_pg"):
        e_tc = rel_vector(tc.get, ref.get, f)
        e_ms = rel_vector(ms.get, ref.get, f)
        assert e_tc <= 3.0 * e_ms + 1e-6, (f, e_tc, e_ms)
        assert rel_vector(tc.get, ms.get, f) <= 1e-4, f


def test_diagnostics_match_numpy():
    from pllcart3d_b200.solver import Solver

    wl = workload("fingering-32x16x16")
    ic = workload_fields(wl)
    s = Solver(wl.params)
    s.load_ic(ic)
    s.step(5)
    d = s.diagnostics()
    p = wl.params
    c = s.get("c_old")[3:p.nx + 3, 1:p.ny + 1, 1:p.nz + 1]
    assert d["mass"] == pytest.approx(c.sum() * p.dx * p.dy * p.dz, rel=1e-12)
    cbar = c.mean(axis=(1, 2))
    assert d["mixing_length"] == pytest.approx(((cbar > 0.01) & (cbar < 0.99)).sum() * p.dx, rel=1e-12)
    u, v, w = (s.get(f"{q}_old") for q in "uvw")
    div = ((u[4:p.nx + 4, 1:p.ny + 1, 1:p.nz + 1] - u[3:p.nx + 3, 1:p.ny + 1, 1:p.nz + 1]) / p.dx
           + (v[3:p.nx + 3, 2:p.ny + 2, 1:p.nz + 1] - v[3:p.nx + 3, 1:p.ny + 1, 1:p.nz + 1]) / p.dy
           + (w[3:p.nx + 3, 1:p.ny + 1, 2:p.nz + 2] - w[3:p.nx + 3, 1:p.ny + 1, 1:p.nz + 1]) / p.dz)
    assert d["div_max"] == pytest.approx(np.abs(div).max(), rel=1e-9, abs=1e-12)


@pytest.mark.parametrize("name", ["fingering-16x128x128", "fingering-8x256x256", "fingering-8x128x256"])
def test_persistent_tcgen05_dct_equals_per_tile(name):
    """The persistent tcgen05 DCT (one CTA per SM, double-buffered TMEM) runs
    every tile with the arithmetic of the one-tile-per-CTA kernel: the whole
    state agrees bit for bit."""
    from pllcart3d_b200.solver import Solver

    wl = workload(name)
    ic = workload_fields(wl)
    a = Solver(wl.params, precision="mixed")
    b = Solver(wl.params, precision="mixed", dct_kernel="umma_tile")
    for s in (a, b):
        s.load_ic(ic)
        s.step(2)
        assert s.status() == 0
    for f in ("phi", "u_new", "v_new", "w_new", "c_new"):
        assert np.array_equal(a.get(f), b.get(f)), f


@pytest.mark.parametrize("name", ["fingering-64x64x64", "fingering-512x16x16", "fingering-16x512x16"])
def test_segmented_line_solves_one_step(name):
    """The precision form's segmented x / y line solves (lines of 64 and
    512 rows, and the one-row-shorter staggered components) against the FP64
    step, next to the precision form's sequential path (exact_dct: Thomas
    sweeps and sequential-order DCT sums): both carry FP32-level errors of
    the same size (large relative to a component that is nearly zero on a
    grid one cell wide in z)."""
    from pllcart3d_b200.solver import Solver

    wl = workload(name)
    ic = workload_fields(wl)
    ref = Solver(wl.params, precision="fp64")
    seg = Solver(wl.params, precision="mixed")
    seq = Solver(wl.params, precision="mixed", exact_dct=True)
    for s in (ref, seg, seq):
        s.load_ic(ic)
        s.step(1)
        assert s.status() == 0
    for f in ("c_new", "u_new", "v_new", "w_new"):
        e_seg = rel_maxnorm(seg.get(f), ref.get(f))
        e_seq = rel_maxnorm(seq.get(f), ref.get(f))
        assert e_seg <= 3.0 * e_seq + 1e-6, (f, e_seg, e_seq)


def test_mixed64_tracks_the_fp64_form():
    """The FP64-state form with FP32 WENO5 weights against the FP64 form
    from the same seed: only the nonlinear weights carry FP32 rounding
    (~1e-7 of each upwind derivative): after 200 steps of the 64x32x32
    case c stays within 1e-6 of the FP64 form and the velocities within
    1e-5 of their vector's max-norm (measured 2.6e-6 in u)."""
    from pllcart3d_b200.solver import Solver

    wl = workload("fingering-64x32x32")
    ic = workload_fields(wl)
    a = Solver(wl.params, precision="fp64")
    b = Solver(wl.params, precision="mixed64")
    for s in (a, b):
        s.load_ic(ic)
        s.step(200)
        assert s.status() == 0
    assert rel_maxnorm(b.get("c_new"), a.get("c_new")) <= 1e-6
    for f in ("u_new", "v_new", "w_new"):
        assert rel_vector(b.get, a.get, f) <= 1e-5, f


def test_tma_explicit_kernel_in_the_precision_form():
    """The TMA-staged plane-marching explicit operator (selectable in the
    precision form, the default of the FP64 forms) computes each cell with
    the per-cell FP32 arithmetic; one step agrees with the paired kernel's to
    FP32 rounding."""
    from pllcart3d_b200.solver import Solver

    wl = workload("fingering-64x64x64")
    ic = workload_fields(wl)
    a = Solver(wl.params, precision="mixed")
    b = Solver(wl.params, precision="mixed", explicit_kernel="tma")
    for s in (a, b):
        s.load_ic(ic)
        s.step(1)
        assert s.status() == 0
    for f in ("c_new", "u_new", "v_new", "w_new"):
        assert rel_vector(b.get, a.get, f) <= 1e-5, f
