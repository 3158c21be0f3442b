"""ctypes front end for the test-only CPU checkers built by oracle/Makefile.

* ``RefRun``    - the reference's own pllcart3d.c step routines, compiled into
                  oracle/_ref/libpllref.so (only present where the reference
                  sources were available at build time);
* ``OracleRun`` - the project's CPU restatement, oracle/liboracle.so.

Test infrastructure only: imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of bench.py, never by the GPU library.
"""

from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libpllref.so")
ORACLE_LIB = os.path.join(HERE, "liboracle.so")

FIELDS = (
    ["c_old", "c_new", "c_hn", "c_hnm1"]
    + [f"{q}_{s}" for q in "uvw" for s in ("old", "new", "hn", "hnm1", "pg")]
    + [f"mu_{t}_{m}" for t in ("old", "new") for m in ("cell", "xy", "xz", "yz")]
    + ["phi", "div"]
)

_D = ctypes.c_double
_I = ctypes.c_int
_P = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_P)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def oracle_available() -> bool:
    return os.path.exists(ORACLE_LIB)


def build(ref: bool = True, ref_dir: str | None = None) -> None:
    """Build liboracle.so, and the reference library when its sources exist
    (in ``ref_dir``, else in the directory PLL_REFERENCE_DIR names)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    ref_dir = ref_dir or os.environ.get("PLL_REFERENCE_DIR")
    if ref and ref_dir and os.path.isfile(os.path.join(ref_dir, "pllcart3d.c")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_dir}"], check=True)


class RefRun:
    """One in-process instance of the compiled reference (global state)."""

    def __init__(self, params, ic=None):
        if not ref_available():
            raise FileNotFoundError(REF_LIB)
        self.lib = lib = ctypes.CDLL(REF_LIB, mode=os.RTLD_LOCAL)
        for name in ("pllref_last_dt", "pllref_tval", "pllref_timestep",
                     "pllref_find_cfl", "pllref_bulk_velo", "pllref_step_dt"):
            getattr(lib, name).restype = _D
        lib.pllref_calculate_weno.restype = _D
        lib.pllref_calculate_weno.argtypes = [_P, _I, _I]
        for name in ("pllref_concentration", "pllref_xmom", "pllref_ymom",
                     "pllref_zmom"):
            getattr(lib, name).argtypes = [_D, _D, _D, _D]
        for name in ("pllref_phisolver", "pllref_velo_correction",
                     "pllref_pressure_gradient"):
            getattr(lib, name).argtypes = [_D, _D, _D]
        lib.pllref_substep.argtypes = [_D, _I]
        self.params = params
        self.shape = params.shape
        self._dir = tempfile.mkdtemp(prefix="pllref_")
        params.write(self._dir)
        if lib.pllref_init(self._dir.encode()) != 0:
            raise RuntimeError("reference init failed")
        if ic is not None:
            self.load_ic(ic)

    def set_fast_dct(self, fast: bool) -> None:
        self.lib.pllref_set_fast_dct(int(bool(fast)))

    def load_ic(self, ic) -> None:
        arrs = [np.ascontiguousarray(ic[k], dtype=np.float64) for k in "cuvw"]
        self.lib.pllref_load_ic(*[_ptr(a) for a in arrs])

    def steps(self, n: int) -> None:
        self.lib.pllref_steps(int(n))

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self.shape, dtype=np.float64)
        if self.lib.pllref_get(name.encode(), _ptr(out)) != 0:
            raise KeyError(name)
        return out

    def set(self, name: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if self.lib.pllref_set(name.encode(), _ptr(a)) != 0:
            raise KeyError(name)

    def state(self) -> dict:
        return {f: self.get(f) for f in FIELDS}

    # ---- the reference's own output routines, writing into `directory` ----
    def write_to_file(self, fileno: int, directory: str) -> None:
        assert self.lib.pllref_write_to_file(int(fileno), directory.encode()) == 0

    def midfield(self, tstep, fileno, tval, outtime, outmid, cavgtime, directory: str) -> None:
        f = self.lib.pllref_midfield
        f.argtypes = [_I, _I, _D, _D, _D, _D, ctypes.c_char_p]
        assert f(int(tstep), int(fileno), tval, outtime, outmid, cavgtime, directory.encode()) == 0

    def intermediate(self, directory: str) -> dict:
        ts, fn, tv, ot = _I(), _I(), _D(), _D()
        assert self.lib.pllref_intermediate(directory.encode(), ctypes.byref(ts), ctypes.byref(fn),
                                            ctypes.byref(tv), ctypes.byref(ot)) == 0
        return {"tstep": ts.value, "fileno": fn.value, "tval": tv.value, "outtime": ot.value}

    def conc_average(self, tval: float, directory: str) -> None:
        f = self.lib.pllref_conc_average
        f.argtypes = [_D, ctypes.c_char_p]
        assert f(tval, directory.encode()) == 0

    def find_wmax(self, tval: float, directory: str) -> None:
        f = self.lib.pllref_find_wmax
        f.argtypes = [_D, ctypes.c_char_p]
        assert f(tval, directory.encode()) == 0

    def find_max(self, directory: str) -> None:
        assert self.lib.pllref_find_max(directory.encode()) == 0

    def shift_conc(self, ampli: float, lamb: float, subharm: int) -> None:
        f = self.lib.pllref_shift_conc
        f.argtypes = [_D, _D, _I]
        f(ampli, lamb, subharm)

    @property
    def dt(self) -> float:
        return self.lib.pllref_last_dt()

    @property
    def timestep(self) -> float:
        return self.lib.pllref_timestep()


class OracleRun:
    """One instance of the CPU restatement (opaque handle, re-entrant)."""

    def __init__(self, params, ic=None):
        if not oracle_available():
            raise FileNotFoundError(ORACLE_LIB)
        self.lib = lib = ctypes.CDLL(ORACLE_LIB, mode=os.RTLD_LOCAL)
        lib.orc_create.restype = ctypes.c_void_p
        lib.orc_create.argtypes = [_P, ctypes.POINTER(_I)]
        lib.orc_destroy.argtypes = [ctypes.c_void_p]
        lib.orc_load_ic.argtypes = [ctypes.c_void_p, _P, _P, _P, _P]
        lib.orc_steps.argtypes = [ctypes.c_void_p, _I]
        lib.orc_field.restype = _P
        lib.orc_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        lib.orc_last_dt.restype = _D
        lib.orc_last_dt.argtypes = [ctypes.c_void_p]
        lib.orc_timestep.restype = _D
        lib.orc_timestep.argtypes = [ctypes.c_void_p]
        lib.orc_step_dt.restype = _D
        lib.orc_step_dt.argtypes = [ctypes.c_void_p]
        lib.orc_bulk_velo.restype = _D
        lib.orc_bulk_velo.argtypes = [ctypes.c_void_p]
        lib.orc_find_cfl.restype = _D
        lib.orc_find_cfl.argtypes = [ctypes.c_void_p]
        lib.orc_substep.argtypes = [ctypes.c_void_p, _D, _I]
        lib.orc_call.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _D, _D, _D, _D]
        lib.orc_call.restype = _I
        lib.orc_set_fast_dct.argtypes = [ctypes.c_void_p, _I]
        self.params = params
        self.shape = params.shape
        dv = np.array(_param_doubles(params), dtype=np.float64)
        iv = (_I * 8)(*_param_ints(params))
        self.h = lib.orc_create(_ptr(dv), iv)
        if not self.h:
            raise RuntimeError("oracle create failed")
        if ic is not None:
            self.load_ic(ic)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.lib.orc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def set_fast_dct(self, fast: bool) -> None:
        self.lib.orc_set_fast_dct(self.h, int(bool(fast)))

    def load_ic(self, ic) -> None:
        arrs = [np.ascontiguousarray(ic[k], dtype=np.float64) for k in "cuvw"]
        self.lib.orc_load_ic(self.h, *[_ptr(a) for a in arrs])

    def steps(self, n: int) -> None:
        self.lib.orc_steps(self.h, int(n))

    def substep(self, dt: float, rk: int) -> None:
        self.lib.orc_substep(self.h, float(dt), int(rk))

    def call(self, routine: str, a=0.0, b=0.0, c=0.0, d=0.0) -> None:
        if self.lib.orc_call(self.h, routine.encode(), a, b, c, d) != 0:
            raise KeyError(routine)

    def view(self, name: str) -> np.ndarray:
        p = self.lib.orc_field(self.h, name.encode())
        if not p:
            raise KeyError(name)
        n = int(np.prod(self.shape))
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(self.shape)

    def get(self, name: str) -> np.ndarray:
        return self.view(name).copy()

    def set(self, name: str, arr: np.ndarray) -> None:
        self.view(name)[...] = arr

    def state(self) -> dict:
        return {f: self.get(f) for f in FIELDS}

    @property
    def dt(self) -> float:
        return self.lib.orc_last_dt(self.h)

    @property
    def timestep(self) -> float:
        return self.lib.orc_timestep(self.h)

    def step_dt(self) -> float:
        return self.lib.orc_step_dt(self.h)

    def bulk_velo(self) -> float:
        return self.lib.orc_bulk_velo(self.h)

    def find_cfl(self) -> float:
        return self.lib.orc_find_cfl(self.h)


def _param_doubles(p):
    return [p.X1, p.X2, p.Y1, p.Y2, p.Z1, p.Z2, p.Re, p.Pe, p.Vratio, p.Fx,
            p.Fy, p.CFLmax, p.Timestep, p.Mum, p.Lambda, 0.0]


def _param_ints(p):
    return [p.Nx_cell_global, p.Ny_cell_global, p.Nz_cell_global, p.Nmvp,
            0, 0, 0, 0]
