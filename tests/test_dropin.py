"""The drop-in layer (libpllcart3d_dropin.so) inside the reference's own
time-step loop and on its own data structures.

Two independent in-process copies of the reference (pllcart3d.c compiled by
oracle/Makefile) start from the same state: one advances with its own
routines, the other with every step routine taken from the drop-in library
(pllref_steps_with), or through the drop-in's resident fast path
(pllgpu_attach / pllgpu_advance / pllgpu_sync_to_host).  Tolerance: 1e-10 of
each field's max-norm, velocity-like fields against their vector's.
"""

import ctypes
import os
import shutil
import tempfile

import numpy as np
import pytest

import oracle.pyref as pyref
from pllcart3d_b200.ic import workload_fields
from pllcart3d_b200.params import workload
from tests.util import STATE_FIELDS, rel_vector

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not pyref.ref_available(), reason="reference not compiled")]

TOL = 1e-10
ROUTINES = ["concentration", "calculate_viscosity", "xmom", "ymom", "zmom",
            "update_velo_boundary", "divergence", "phisolver_dct", "update_phi_ghosts",
            "velo_correction", "update_veloghost_points", "pressure_gradient",
            "update_old_conc", "update_old_velo", "update_old_visc", "find_cfl", "bulk_velo"]


def _second_reference(params, ic):
    """A RefRun on a copy of the library: its own globals and arrays."""
    d = tempfile.mkdtemp(prefix="pllref2_")
    path = os.path.join(d, "libpllref_copy.so")
    shutil.copy(pyref.REF_LIB, path)
    saved = pyref.REF_LIB
    pyref.REF_LIB = path
    try:
        return pyref.RefRun(params, ic)
    finally:
        pyref.REF_LIB = saved


def _dropin(params, timestep):
    from pllcart3d_b200 import _lib

    L = ctypes.CDLL(_lib.DROPIN_PATH, mode=os.RTLD_LOCAL)
    ints = {"Nx_cell_global": params.nx, "Ny_cell_global": params.ny,
            "Nz_cell_global": params.nz, "Nx_ghost": 3, "Ny_ghost": 1, "Nz_ghost": 1,
            "Nmvp": params.Nmvp}
    dbls = {"X1": params.X1, "X2": params.X2, "Y1": params.Y1, "Y2": params.Y2,
            "Z1": params.Z1, "Z2": params.Z2, "Re": params.Re, "Pe": params.Pe,
            "Vratio": params.Vratio, "M": params.Vratio, "Vnorm": 0.0, "Fx": params.Fx,
            "Fy": params.Fy, "CFLmax": params.CFLmax, "Timestep": timestep,
            "Mum": params.Mum, "Lambda": params.Lambda}
    for k, v in ints.items():
        ctypes.c_int.in_dll(L, k).value = v
    for k, v in dbls.items():
        ctypes.c_double.in_dll(L, k).value = v
    L.pllgpu_dropin_status.restype = ctypes.c_int
    return L


def _compare(a, b):
    for f in STATE_FIELDS:
        e = rel_vector(a.get, b.get, f)
        assert e <= TOL, f"{f}: {e:.3e}"


@pytest.mark.parametrize("name,kw", [("fingering-24x12x12", {}),
                                     ("fingering-20x8x10", {"Fx": 1.0, "Fy": -0.5})])
def test_dropin_routines_in_reference_loop(name, kw):
    wl = workload(name)
    wl.params = wl.params.replace(**kw)
    ic = workload_fields(wl)
    a = pyref.RefRun(wl.params, ic)
    b = _second_reference(wl.params, ic)
    L = _dropin(wl.params, b.timestep)
    table = (ctypes.c_void_p * len(ROUTINES))(
        *[ctypes.cast(getattr(L, n), ctypes.c_void_p).value for n in ROUTINES])
    steps = 3
    a.steps(steps)
    b.lib.pllref_steps_with.argtypes = [ctypes.c_int, ctypes.c_void_p]
    b.lib.pllref_steps_with(steps, table)
    assert L.pllgpu_dropin_status() == 0
    _compare(b, a)
    L.pllgpu_finalize()


def test_dropin_resident_fast_path():
    wl = workload("fingering-24x12x12")
    ic = workload_fields(wl)
    a = pyref.RefRun(wl.params, ic)
    b = _second_reference(wl.params, ic)
    L = _dropin(wl.params, b.timestep)
    s = (ctypes.c_void_p * 8)()
    b.lib.pllref_structs(s)
    L.pllgpu_attach.argtypes = [ctypes.c_void_p] * 8
    L.pllgpu_advance.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    assert L.pllgpu_attach(*[s[i] for i in range(8)]) == 0
    tval = ctypes.c_double(0.0)
    assert L.pllgpu_advance(5, ctypes.byref(tval)) == 0
    assert L.pllgpu_sync_to_host() == 0
    a.steps(5)
    assert tval.value == pytest.approx(a.lib.pllref_tval(), rel=1e-12)
    _compare(b, a)
    L.pllgpu_finalize()


class _Tds(ctypes.Structure):
    _fields_ = [("acof", ctypes.POINTER(ctypes.c_double)), ("bcof", ctypes.POINTER(ctypes.c_double)),
                ("ccof", ctypes.POINTER(ctypes.c_double)), ("rhs", ctypes.POINTER(ctypes.c_double))]


def _triple(arr):
    """double*** view of a C-contiguous (n0, n1, n2) array (keeps refs)."""
    n0, n1, _ = arr.shape
    P = ctypes.POINTER(ctypes.c_double)
    rows = []
    top = (ctypes.POINTER(P) * n0)()
    for i in range(n0):
        mid = (P * n1)()
        for j in range(n1):
            mid[j] = arr[i, j].ctypes.data_as(P)
        rows.append(mid)
        top[i] = ctypes.cast(mid, ctypes.POINTER(P))
    return top, rows


def test_dropin_line_solvers_weno_and_dct():
    wl = workload("fingering-16x8x8")
    ic = workload_fields(wl)
    ref = pyref.RefRun(wl.params, ic)
    L = _dropin(wl.params, ref.timestep)
    P = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(9)
    # pll_tridiag on Tds structures, against the reference's own
    N, n = 7, 13
    a = rng.uniform(-1, -0.1, (N, n)); c = rng.uniform(-1, -0.1, (N, n))
    b = 3 + rng.uniform(0, 1, (N, n)); r = rng.standard_normal((N, n))
    mine = [x.copy() for x in (a, b, c, r)]
    theirs = [x.copy() for x in (a, b, c, r)]
    tds = (_Tds * N)(*[_Tds(*(m[s].ctypes.data_as(P) for m in mine)) for s in range(N)])
    L.pll_tridiag.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.pll_tridiag(tds, N, n)
    ref.lib.pllref_pll_tridiag.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, P]
    ref.lib.pllref_pll_tridiag(N, n, *(t.ctypes.data_as(P) for t in theirs))
    for m, t in zip(mine[1:], theirs[1:]):
        assert np.array_equal(m, t)
    # tridiag_1rhs
    x1, x2 = r[0].copy(), r[0].copy()
    L.tridiag_1rhs.argtypes = [ctypes.c_int, P, P, P, P]
    ref.lib.pllref_tridiag_1rhs.argtypes = [ctypes.c_int, P, P, P, P]
    L.tridiag_1rhs(n, a[0].ctypes.data_as(P), b[0].ctypes.data_as(P), c[0].ctypes.data_as(P), x1.ctypes.data_as(P))
    ref.lib.pllref_tridiag_1rhs(n, a[0].ctypes.data_as(P), b[0].ctypes.data_as(P), c[0].ctypes.data_as(P),
                                x2.ctypes.data_as(P))
    assert np.array_equal(x1, x2)
    # calculate_weno
    d1 = rng.standard_normal(12)
    L.calculate_weno.restype = ctypes.c_double
    L.calculate_weno.argtypes = [P, ctypes.c_int, ctypes.c_int]
    for kk, sign in ((3, 1), (8, -1)):
        assert L.calculate_weno(d1.ctypes.data_as(P), kk, sign) == \
            ref.lib.pllref_calculate_weno(d1.ctypes.data_as(P), kk, sign)
    # fdct_3d / idct_3d on double*** [ndim1][ndim2][nt] (fftw_3d.h:45-106)
    ny, nz, nx = wl.params.ny, wl.params.nz, wl.params.nx
    src = rng.standard_normal((ny, nz, nx))
    out = np.zeros_like(src)
    tin, k1 = _triple(src)
    tout, k2 = _triple(out)
    L.plan_dct_3d(ny, nz, nx)
    L.fdct_3d(ny, nz, nx, tin, tout)
    x = np.transpose(src, (2, 1, 0))           # [nt][ndim2][ndim1]
    j = np.arange(ny); k = np.arange(nz)
    Cy = 2 * np.cos(np.pi * (2 * j[None, :] + 1) * j[:, None] / (2 * ny))
    Cz = 2 * np.cos(np.pi * (2 * k[None, :] + 1) * k[:, None] / (2 * nz))
    want = np.einsum("ab,tbc,dc->tad", Cz, x, Cy)
    assert np.allclose(np.transpose(out, (2, 1, 0)), want, rtol=1e-12, atol=1e-11)
    back = np.zeros_like(src)
    tb, k3 = _triple(back)
    L.idct_3d(ny, nz, nx, tout, tb)
    assert np.allclose(back, src, rtol=1e-12, atol=1e-12)
    assert L.pllgpu_dropin_status() == 0
    L.pllgpu_finalize()


def _abc_all(run, ranges):
    """Every variable's Ax/Ay/Az triples on its unknown range, from the
    reference's Tri_abc arrays (NaN elsewhere)."""
    out = {}
    lib = run.lib
    P = ctypes.POINTER(ctypes.c_double)
    lib.pllref_get_abc.argtypes = [ctypes.c_char_p] + [ctypes.c_int] * 6 + [P] * 3
    for var, q in enumerate("cuvw"):
        r = ranges[var]
        for ax in ("Ax", "Ay", "Az"):
            a, b, c = (np.full(run.shape, np.nan) for _ in range(3))
            assert lib.pllref_get_abc(f"{q}_{ax}".encode(), *r, *(pyref._ptr(t) for t in (a, b, c))) == 0
            sl = tuple(slice(r[2 * d], r[2 * d + 1] + 1) for d in range(3))
            out[f"{q}_{ax}"] = np.stack([a[sl], b[sl], c[sl]])
    return out


@pytest.mark.parametrize("name,kw", [("fingering-20x8x10", {}), ("fingering-18x9x7", {"Nmvp": 1, "Vratio": 1.0})])
def test_dropin_acoef_fills_reference_tri_abc(name, kw):
    """The drop-in A_conc / A_umom / A_vmom / A_wmom (pllcart3d.c:1411-1536)
    fill the caller's Tri_abc arrays with the reference's own coefficients:
    both are called on the same reference structures after two steps, from
    the old and from the new viscosity; every triple on each variable's
    unknown range agrees to 1e-14 of the largest coefficient."""
    wl = workload(name)
    wl.params = wl.params.replace(**kw)
    ic = workload_fields(wl)
    a = pyref.RefRun(wl.params, ic)
    a.steps(2)
    L = _dropin(wl.params, a.timestep)
    fns = ["A_conc", "A_umom", "A_vmom", "A_wmom"]
    table = (ctypes.c_void_p * 4)(*[ctypes.cast(getattr(L, n), ctypes.c_void_p).value for n in fns])
    a.lib.pllref_acoef_with.argtypes = [ctypes.c_void_p, ctypes.c_int]
    a.lib.pllref_range.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    ranges = []
    for var in range(4):
        r = (ctypes.c_int * 6)()
        a.lib.pllref_range(var, r)
        ranges.append(list(r))
    for mu_which in (0, 1):
        assert a.lib.pllref_acoef_with(None, mu_which) == 0
        want = _abc_all(a, ranges)
        assert a.lib.pllref_acoef_with(table, mu_which) == 0
        assert L.pllgpu_dropin_status() == 0
        got = _abc_all(a, ranges)
        for key, w in want.items():
            g = got[key]
            assert np.isfinite(w).all() and np.isfinite(g).all(), key
            err = float(np.abs(g - w).max() / np.abs(w).max())
            assert err <= 1e-14, (key, mu_which, err)
    L.pllgpu_finalize()
