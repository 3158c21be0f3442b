"""``Params.read`` parses param.input files to the values the reference's
own ``input()`` (pllcart3d.c:271-350, compiled by oracle/Makefile) reads
from them: a file written by ``Params.write`` with values off every default,
and, where PLL_REFERENCE_DIR names the reference's source directory, the
param.input the reference ships."""

import ctypes
import dataclasses
import os
import shutil
import tempfile

import numpy as np
import pytest

import oracle.pyref as pyref
from pllcart3d_b200.params import PARAM_FIELDS, Params

pytestmark = pytest.mark.skipif(not pyref.ref_available(), reason="reference library not built")


def _reference_reads(path):
    """input() of a private copy of the reference library on `path`."""
    d = tempfile.mkdtemp(prefix="pllparam_")
    lib_path = os.path.join(d, "libpllref_param.so")
    shutil.copy(pyref.REF_LIB, lib_path)
    run = os.path.join(d, "run")
    os.mkdir(run)
    shutil.copy(path, os.path.join(run, "param.input"))
    lib = ctypes.CDLL(lib_path, mode=os.RTLD_LOCAL)
    out = np.zeros(34)
    lib.pllref_read_input.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
    assert lib.pllref_read_input(run.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 34
    return out


def _as_vector(p: Params):
    return np.array([float(getattr(p, name)) for name, _, _ in PARAM_FIELDS])


def test_written_file_reads_back_as_the_reference_reads_it(tmp_path):
    vals = {}
    for n, (name, typ, _) in enumerate(PARAM_FIELDS):
        vals[name] = (7 + n) if typ is int else 0.125 * (n + 1) - 1.0 / 3.0
    vals.update(Nx_cell_global=40, Ny_cell_global=12, Nz_cell_global=10, Nx_ghost=3, Ny_ghost=1, Nz_ghost=1,
                Nmvp=1, Wavpert=0, Subharm=1)
    p = Params(**vals)
    path = p.write(str(tmp_path))
    got = Params.read(path)
    assert dataclasses.asdict(got) == dataclasses.asdict(p)
    np.testing.assert_array_equal(_as_vector(got), _reference_reads(path))


def test_shipped_param_input():
    ref_dir = os.environ.get("PLL_REFERENCE_DIR")
    path = os.path.join(ref_dir, "param.input") if ref_dir else ""
    if not os.path.isfile(path):
        pytest.skip("PLL_REFERENCE_DIR does not name the reference's source directory")
    got = Params.read(path)
    np.testing.assert_array_equal(_as_vector(got), _reference_reads(path))
    # the shipped run: the non-monotonic viscosity law
    assert got.Nmvp == 1
