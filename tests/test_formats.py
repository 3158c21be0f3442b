"""The CPU restatement of the reference's output formats (oracle/formats.py)
against the files the compiled reference itself writes, on a reference state
after a few steps."""

import os
import tempfile

import numpy as np
import pytest

from oracle import formats, pyref
from pllcart3d_b200.ic import workload_fields
from pllcart3d_b200.params import workload

pytestmark = pytest.mark.skipif(not pyref.ref_available(), reason="reference library not built")


@pytest.fixture(scope="module")
def ref_state():
    wl = workload("fingering-16x8x8")
    ref = pyref.RefRun(wl.params, workload_fields(wl))
    ref.steps(6)
    return ref, ref.state()


def _read(d, name, mode="rb"):
    with open(os.path.join(d, name), mode) as f:
        return f.read()


def test_snapshot_bytes(ref_state):
    ref, st = ref_state
    with tempfile.TemporaryDirectory() as d:
        ref.write_to_file(7, d)
        got = _read(d, "caf0007R000.bin")
    assert got == formats.snapshot(st["u_new"], st["v_new"], st["w_new"], st["c_new"])
    assert len(got) == 16 * 16 * 8 * 8


def test_restart_bytes_and_round_trip(ref_state):
    ref, st = ref_state
    with tempfile.TemporaryDirectory() as d:
        ref.midfield(12, 3, 0.125, 0.5, 0.75, 0.25, d)
        assert _read(d, "middata", "r") == formats.middata(12, 3, 0.125, 0.5, 0.75, 0.25)
        data = _read(d, "midfield000.bin")
        assert data == formats.midfield(st)
        back = formats.read_midfield(data, st["c_old"].shape)
        for f in formats.MID_FIELDS:
            assert np.array_equal(back[f], st[f]), f
        meta = ref.intermediate(d)
    assert meta == {"tstep": 12, "fileno": 3, "tval": 0.125, "outtime": 0.5}


def test_conc_average_bytes(ref_state):
    ref, st = ref_state
    with tempfile.TemporaryDirectory() as d:
        ref.conc_average(0.375, d)
        ref.conc_average(0.5, d)
        y, z, yz = formats.conc_average(st["c_new"], 0.375)
        y2, z2, yz2 = formats.conc_average(st["c_new"], 0.5)
        assert _read(d, "cavgy.bin") == y + y2
        assert _read(d, "cavgz.bin") == z + z2
        assert _read(d, "cavgyz.bin") == yz + yz2


def test_wmax_and_find_max(ref_state):
    ref, st = ref_state
    with tempfile.TemporaryDirectory() as d:
        ref.find_wmax(0.25, d)
        assert _read(d, "wmax.bin") == formats.wmax_record(st["w_new"], 0.25)
        ref.find_max(d)
        text = _read(d, "Outscreen", "r")
    assert text.endswith(formats.find_max_text(st["u_new"], st["v_new"], st["w_new"], st["c_new"]))
