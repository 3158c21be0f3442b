"""The device-packed output files (pllgpu_write_snapshot, _write_restart,
_read_restart, _conc_average, _find_wmax, _find_max) byte for byte against
the files the compiled reference writes from the same state, and against the
CPU restatement where the reference's branch is out of reach (the even-cell
subsample above 2e7 cells)."""

import ctypes
import os
import tempfile

import numpy as np
import pytest

from oracle import formats, pyref
from pllcart3d_b200.ic import workload_fields
from pllcart3d_b200.params import workload

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not pyref.ref_available(), reason="reference library not built")]

STATE = ("c_old", "c_new", "c_hn", "c_hnm1", "u_old", "u_new", "u_hnm1", "u_pg", "v_old", "v_new",
         "v_hnm1", "v_pg", "w_old", "w_new", "w_hnm1", "w_pg")


@pytest.fixture(scope="module")
def pair(tmp_path_factory):
    """A reference state after 6 steps, every reference output file written
    from it (into `refdir`, before anything else can re-initialise the
    reference's global state), and a GPU context holding the same state."""
    from pllcart3d_b200.solver import Solver

    wl = workload("fingering-16x8x8")
    ref = pyref.RefRun(wl.params, workload_fields(wl))
    ref.steps(6)
    st = ref.state()
    refdir = str(tmp_path_factory.mktemp("refout"))
    ref.write_to_file(5, refdir)
    ref.midfield(40, 2, 0.3125, 0.5, 0.625, 0.375, refdir)
    for t in (0.25, 0.5):
        ref.conc_average(t, refdir)
    ref.find_wmax(0.75, refdir)
    ref.find_max(refdir)
    gpu = Solver(wl.params)
    gpu.load_ic(workload_fields(wl))
    for f in STATE:
        gpu.set(f, st[f])
    return wl, refdir, st, gpu


def _read(d, name, mode="rb"):
    with open(os.path.join(d, name), mode) as f:
        return f.read()


def test_snapshot_matches_reference(pair):
    wl, a, st, gpu = pair
    with tempfile.TemporaryDirectory() as b:
        gpu.write_snapshot(5, b)
        assert _read(b, "caf0005R000.bin") == _read(a, "caf0005R000.bin")


def test_snapshot_even_cell_subsample(pair):
    wl, a, st, gpu = pair
    with tempfile.TemporaryDirectory() as d:
        gpu.write_snapshot(1, d, subsample=True)
        got = _read(d, "caf0001R000.bin")
    assert got == formats.snapshot(st["u_new"], st["v_new"], st["w_new"], st["c_new"], subsample=True)


def test_restart_write_read_round_trip(pair):
    from pllcart3d_b200.solver import Solver

    wl, a, st, gpu = pair
    with tempfile.TemporaryDirectory() as b:
        gpu.write_restart(40, 2, 0.3125, 0.5, 0.625, 0.375, b)
        assert _read(b, "middata", "r") == _read(a, "middata", "r")
        assert _read(b, "midfield000.bin") == _read(a, "midfield000.bin")
        # a fresh context restarts from the reference's files
        other = Solver(wl.params)
        meta = other.read_restart(a)
    assert meta == {"tstep": 40, "fileno": 2, "tval": 0.3125, "outtime": 0.5}
    for f in formats.MID_FIELDS:
        assert np.array_equal(other.get(f), st[f]), f


def test_restart_then_steps_match_reference():
    """Restart the reference and the GPU from the same midfield files and
    step both: the restart start-up (viscosity of c_old) is the reference's."""
    from pllcart3d_b200.solver import Solver

    wl = workload("fingering-16x8x8")
    a = pyref.RefRun(wl.params, workload_fields(wl))
    a.steps(4)
    with tempfile.TemporaryDirectory() as d:
        a.midfield(4, 1, 0.0, 0.0, 0.0, 0.0, d)
        b = pyref.RefRun(wl.params)
        meta = b.intermediate(d)
        b.lib.pllref_restart_startup.argtypes = [ctypes.c_double]
        assert b.lib.pllref_restart_startup(meta["tval"]) == 0
        g = Solver(wl.params)
        g.read_restart(d)
    b.steps(5)
    g.step(5)
    for f in ("c_new", "u_new", "v_new", "w_new"):
        ref = b.get(f)
        assert np.abs(g.get(f) - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), f


def test_conc_average_wmax_find_max(pair):
    wl, a, st, gpu = pair
    with tempfile.TemporaryDirectory() as b:
        for t in (0.25, 0.5):
            gpu.conc_average(t, b)
        for name in ("cavgy.bin", "cavgz.bin", "cavgyz.bin"):
            assert _read(b, name) == _read(a, name), name
        w = gpu.find_wmax(0.75, b)
        assert _read(b, "wmax.bin") == _read(a, "wmax.bin")
        assert w == pytest.approx(max(0.0, st["w_new"][3:-3, 1:-1, 1:-1].max()), abs=0)
        gpu.find_max(b)
        assert _read(b, "Outscreen", "r") == _read(a, "Outscreen", "r")


def test_find_max_reports_nan_without_exit(pair):
    from pllcart3d_b200 import _lib

    wl, a, st, gpu = pair
    bad = st["c_new"].copy()
    bad[5, 3, 4] = np.nan
    gpu.set("c_new", bad)
    with tempfile.TemporaryDirectory() as d:
        with pytest.raises(_lib.PllGpuError):
            gpu.find_max(d)
        assert _read(d, "Outscreen", "r") == "nan in b 5 3 4 \n"
    gpu.clear_status()
    gpu.set("c_new", st["c_new"])


def test_precision_form_outputs_close():
    from pllcart3d_b200.solver import Solver

    wl = workload("fingering-16x8x8")
    ic = workload_fields(wl)
    s = Solver(wl.params, precision="mixed")
    s.load_ic(ic)
    s.step(3)
    with tempfile.TemporaryDirectory() as d:
        s.write_snapshot(0, d)
        got = np.frombuffer(_read(d, "caf0000R000.bin"), dtype=np.float32)
    want = np.frombuffer(formats.snapshot(s.get("u_new"), s.get("v_new"), s.get("w_new"), s.get("c_new")),
                         dtype=np.float32)
    assert np.array_equal(got, want)
