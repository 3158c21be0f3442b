"""Host-side front end of the GPU step: the reference's step routines as
methods of a resident-state solver.

``Solver`` owns one ``pllgpu_ctx`` (device state in HBM).  Its methods carry
the names of the reference routines they replace (pllcart3d.c) and run them
on the GPU against the resident state; ``step(n)`` runs whole time steps
(pllcart3d.c:158-195) as CUDA-graph replays.  Fields are numpy float64
arrays over the padded box ``(nx+6, ny+2, nz+2)`` in the reference's
``[i][j][k]`` order.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .params import Params

RK1 = (8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0)   # global_variables.h:17
RK2 = (0.0, -17.0 / 60.0, -5.0 / 12.0)      # global_variables.h:18


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


PRECISIONS = {"fp64": 0, "mixed": 1, "mixed64": 2}


class Solver:
    """precision="fp64": the reference's FP64 arithmetic; "mixed": FP32 state
    and stencils, split-TF32 tensor-core DCT, FP64 Poisson mode solve and
    reductions; "mixed64": the FP64 form with the WENO5 weights in FP32.
    dct_kernel="auto" runs the precision form's DCT passes as
    tcgen05 GEMMs where the plane shape allows (ny, nz in {128, 256}; a
    persistent kernel, one CTA per SM), "umma_tile" the same tcgen05 pass
    with one tile per CTA, "mma_sync" the warp-level split-TF32 GEMM.
    explicit_kernel="auto" runs the explicit operator as the TMA-staged
    plane-marching kernel in the FP64 forms and on FP32x2 cell pairs in the
    precision form; "direct" the per-cell (FP64) / paired (FP32) kernel,
    "tma" the TMA-staged kernel in either form.
    exact_dct=True sums the DCTs in sequential order and, in the precision
    form, runs every line and mode solve as the sequential Thomas sweep (the
    default: the partitioned line solves and, with the tcgen05 DCT, the
    FP32-scratch mode solve)."""

    def __init__(self, params: Params, device: int = 0, exact_dct: bool = False,
                 use_graph: bool = True, precision: str = "fp64", dct_kernel: str = "auto",
                 explicit_kernel: str = "auto"):
        p = self.c_params(params, exact_dct, use_graph, precision, dct_kernel, explicit_kernel)
        self.params = params
        self.precision = precision
        self._L = _lib.lib()
        self._owned = True
        self._h = self._L.pllgpu_create(ctypes.byref(p), int(device))
        if not self._h:
            raise _lib.PllGpuError(2, "pllgpu_create")
        self.shape = params.shape

    @classmethod
    def view(cls, handle, params: Params, precision: str) -> "Solver":
        """A Solver over a context owned elsewhere (an ensemble member)."""
        s = cls.__new__(cls)
        s.params, s.precision, s._L, s._owned, s._h = params, precision, _lib.lib(), False, handle
        s.shape = params.shape
        return s

    @staticmethod
    def c_params(params: Params, exact_dct: bool = False, use_graph: bool = True,
                 precision: str = "fp64", dct_kernel: str = "auto", explicit_kernel: str = "auto"):
        """The pllgpu_params struct of a run."""
        params.validate()
        p = _lib.Params()
        p.nx, p.ny, p.nz = params.nx, params.ny, params.nz
        p.nmvp = params.Nmvp
        p.X1, p.X2, p.Y1, p.Y2, p.Z1, p.Z2 = (params.X1, params.X2, params.Y1,
                                              params.Y2, params.Z1, params.Z2)
        p.Re, p.Pe, p.Vratio = params.Re, params.Pe, params.Vratio
        p.Fx, p.Fy, p.CFLmax = params.Fx, params.Fy, params.CFLmax
        p.Timestep, p.Mum, p.Lambda = params.Timestep, params.Mum, params.Lambda
        p.precision = PRECISIONS[precision]
        p.exact_dct = int(bool(exact_dct))
        p.use_graph = int(bool(use_graph))
        p.dct_kernel = {"auto": 0, "mma_sync": 1, "umma_tile": 2}[dct_kernel]
        p.explicit_kernel = {"auto": 0, "direct": 1, "tma": 2}[explicit_kernel]
        return p

    # ---- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                self._L.pllgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, code: int, what: str) -> None:
        if code != 0:
            raise _lib.PllGpuError(code, what)

    # ---- state ------------------------------------------------------------
    def set(self, name: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != self.shape:
            raise ValueError(f"{name}: shape {a.shape} != {self.shape}")
        fid = _lib.FIELD_NAMES.index(name)
        self._check(self._L.pllgpu_set_field(self._h, fid, _dp(a)), f"set {name}")

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        fid = _lib.FIELD_NAMES.index(name)
        self._check(self._L.pllgpu_get_field(self._h, fid, _dp(out)), f"get {name}")
        return out

    def state(self, names=None) -> dict:
        return {n: self.get(n) for n in (names or _lib.FIELD_NAMES)}

    def load_ic(self, ic: dict) -> None:
        """Initial fields into the *_new arrays, then the start-up of
        pllcart3d.c:81-83 and 126-154."""
        for k in "cuvw":
            self.set(f"{k}_new", ic[k])
        self._check(self._L.pllgpu_start(self._h), "start")

    # ---- time stepping ----------------------------------------------------
    def step(self, n: int = 1) -> None:
        self._check(self._L.pllgpu_steps(self._h, int(n)), "steps")

    @property
    def dt(self) -> float:
        return self._L.pllgpu_last_dt(self._h)

    @property
    def timestep(self) -> float:
        return self._L.pllgpu_timestep(self._h)

    @property
    def tval(self) -> float:
        return self._L.pllgpu_tval(self._h)

    @property
    def kernels_per_step(self) -> int:
        return self._L.pllgpu_kernels_per_step(self._h)

    def diagnostics(self) -> dict:
        """FP64 mass, max |div u|, L2 |div u| and mixing length of the state."""
        out = (ctypes.c_double * 4)()
        self._check(self._L.pllgpu_diagnostics(self._h, out), "diagnostics")
        return {"mass": out[0], "div_max": out[1], "div_l2": out[2], "mixing_length": out[3]}

    # ---- the reference's output files (write_to_file, midfield, ...) --------
    def write_snapshot(self, fileno: int, directory: str = ".", subsample=None) -> None:
        """write_to_file, pllcart3d.c:3047: caf%04dR000.bin in `directory`;
        subsample None follows the reference's 2e7-cell rule."""
        sub = -1 if subsample is None else int(bool(subsample))
        self._check(self._L.pllgpu_write_snapshot_ex(self._h, int(fileno), 0, directory.encode(), sub),
                    "write_snapshot")

    def write_restart(self, tstep: int, fileno: int, tval: float, outtime: float, outmid: float,
                      cavgtime: float, directory: str = ".") -> None:
        """midfield, pllcart3d.c:3121: middata + midfield000.bin."""
        self._check(self._L.pllgpu_write_restart(self._h, int(tstep), int(fileno), float(tval),
                                                 float(outtime), float(outmid), float(cavgtime),
                                                 directory.encode()), "write_restart")

    def read_restart(self, directory: str = ".") -> dict:
        """intermediate, pllcart3d.c:3181, then the restart start-up."""
        ts, fn = ctypes.c_int(), ctypes.c_int()
        tv, ot = ctypes.c_double(), ctypes.c_double()
        self._check(self._L.pllgpu_read_restart(self._h, directory.encode(), ctypes.byref(ts),
                                                ctypes.byref(fn), ctypes.byref(tv), ctypes.byref(ot)),
                    "read_restart")
        self._check(self._L.pllgpu_resume(self._h, tv.value), "resume")
        return {"tstep": ts.value, "fileno": fn.value, "tval": tv.value, "outtime": ot.value}

    def conc_average(self, tval: float, directory: str = ".") -> None:
        """conc_average, pllcart3d.c:3635: appends cavgy/cavgz/cavgyz.bin."""
        self._check(self._L.pllgpu_conc_average(self._h, float(tval), directory.encode()), "conc_average")

    def find_wmax(self, tval: float, directory=None) -> float:
        """find_wmax, pllcart3d.c:3606 (appends wmax.bin when a directory is given)."""
        out = ctypes.c_double()
        d = directory.encode() if directory is not None else None
        self._check(self._L.pllgpu_find_wmax(self._h, float(tval), d, ctypes.byref(out)), "find_wmax")
        return out.value

    def find_max(self, directory=None) -> dict:
        """find_max, pllcart3d.c:3539: max |u|,|v|,|w|,|c| (signed value at
        the last index attaining it) and where; appends to Outscreen when a
        directory is given.  A NaN in c raises PllGpuError (ENAN)."""
        val = (ctypes.c_double * 4)()
        loc = (ctypes.c_int * 12)()
        d = directory.encode() if directory is not None else None
        self._check(self._L.pllgpu_find_max(self._h, d, val, loc), "find_max")
        return {q: (val[n], tuple(loc[3 * n:3 * n + 3])) for n, q in enumerate("uvwc")}

    def shift_conc(self, ampli=None, lamb=None, subharm=None) -> None:
        """shift_conc, pllcart3d.c:3231: the spanwise wave perturbation of
        c_old (defaults: the run's Ampli, Lamb, Subharm)."""
        p = self.params
        a = p.Ampli if ampli is None else ampli
        lm = p.Lamb if lamb is None else lamb
        sh = p.Subharm if subharm is None else subharm
        self._check(self._L.pllgpu_shift_conc(self._h, float(a), float(lm), int(sh)), "shift_conc")

    # ---- state exchange (learned surrogate, judges) -------------------------
    def copy_state_from(self, other: "Solver") -> None:
        """pllgpu_copy_state: this context takes other's whole state."""
        self._check(self._L.pllgpu_copy_state(self._h, other._h), "copy_state")

    def pack_cells(self, d_ptr: int) -> None:
        """Cell-centred (u, v, w, c) float32 [nx][ny][nz][4] into device memory."""
        self._check(self._L.pllgpu_pack_cells(self._h, ctypes.c_void_p(d_ptr)), "pack_cells")

    def unpack_cells(self, d_ptr: int) -> None:
        self._check(self._L.pllgpu_unpack_cells(self._h, ctypes.c_void_p(d_ptr)), "unpack_cells")

    def project(self) -> None:
        """The DCT pressure projection of the *_new velocities (divergence,
        phisolver_dct, velo_correction with its outflow flux fix, ghost
        fills), then mu from c_new and the new -> old rotation: the state a
        step starts from.  With dt*alpha = 1 the correction is u - grad
        lap^-1 div u whatever the time step."""
        self._routine("divergence")
        self._routine("phisolver", 1.0, 1.0, 0.0)
        self._routine("phi_ghosts")
        self._routine("velo_correction", 1.0, 1.0, 0.0)
        self._routine("velo_ghosts")
        self._routine("viscosity_new")
        self._routine("rotate")

    def autotune(self, trial_steps: int = 2) -> int:
        """pllgpu_autotune: picks the fastest launch shapes on steps of this
        run (bit-identical variants); returns the steps it advanced."""
        done = ctypes.c_int()
        self._check(self._L.pllgpu_autotune(self._h, int(trial_steps), ctypes.byref(done)), "autotune")
        return done.value

    def tuning(self) -> tuple:
        e, l = ctypes.c_int(), ctypes.c_int()
        self._check(self._L.pllgpu_tuning(self._h, ctypes.byref(e), ctypes.byref(l)), "tuning")
        return e.value, l.value

    def set_tuning(self, explicit_variant: int, line_variant: int) -> None:
        self._check(self._L.pllgpu_set_tuning(self._h, int(explicit_variant), int(line_variant)),
                    "set_tuning")

    def status(self) -> int:
        return self._L.pllgpu_status(self._h)

    def clear_status(self) -> None:
        self._L.pllgpu_clear_status(self._h)

    # ---- reference routines, one at a time ---------------------------------
    def _routine(self, name: str, *scal) -> float:
        vin = (ctypes.c_double * 4)(*(list(scal) + [0.0] * (4 - len(scal))))
        vout = (ctypes.c_double * 4)()
        self._check(self._L.pllgpu_routine(self._h, _lib.ROUTINES[name], vin, vout), name)
        return vout[0]

    def concentration(self, dt, g, r, vbulk):
        """pllcart3d.c:555-719 (advecting velocities: u/v/w_new)."""
        self._routine("concentration", dt, g, r, vbulk)

    def calculate_viscosity(self):
        """pllcart3d.c:843-886 of c_new into mu_new (889-948 when Nmvp=1)."""
        self._routine("viscosity_new")

    def xmom(self, dt, g, r, vbulk):
        self._routine("xmom", dt, g, r, vbulk)

    def ymom(self, dt, g, r, vbulk):
        self._routine("ymom", dt, g, r, vbulk)

    def zmom(self, dt, g, r, vbulk):
        self._routine("zmom", dt, g, r, vbulk)

    def update_velo_boundary(self):
        self._routine("velo_ghosts")

    update_veloghost_points = update_velo_boundary

    def divergence(self):
        self._routine("divergence")

    def phisolver_dct(self, dt, g, r):
        self._routine("phisolver", dt, g, r)

    def update_phi_ghosts(self):
        self._routine("phi_ghosts")

    def velo_correction(self, dt, g, r):
        self._routine("velo_correction", dt, g, r)

    def pressure_gradient(self, dt, g, r):
        self._routine("pressure_gradient", dt, g, r)

    def update_old(self):
        """update_old_conc / update_old_velo / update_old_visc."""
        self._routine("rotate")

    def bulk_velo(self) -> float:
        return self._routine("bulk_velo")

    def find_cfl(self) -> float:
        return self._routine("find_cfl")

    def substep(self, dt, rk):
        self._routine("substep", dt, float(rk))


def tridiag_batch(a, b, c, r):
    """pll_tridiag (pll_tridiag.c:152) on the GPU for N systems of length n
    (arrays shaped (N, n)); returns (b, c, r) as the reference leaves them."""
    L = _lib.lib()
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.array(b, dtype=np.float64, order="C")
    c = np.array(c, dtype=np.float64, order="C")
    r = np.array(r, dtype=np.float64, order="C")
    N, n = a.shape
    code = L.pllgpu_tridiag_batch(N, n, _dp(a), _dp(b), _dp(c), _dp(r))
    if code:
        raise _lib.PllGpuError(code, "tridiag_batch")
    return b, c, r


def dct2d_batch(kind: int, x: np.ndarray) -> np.ndarray:
    """FFTW REDFT10 (kind 0) / REDFT01 (kind 1) over the last two axes."""
    L = _lib.lib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    howmany = int(np.prod(x.shape[:-2])) if x.ndim > 2 else 1
    n0, n1 = x.shape[-2:]
    out = np.empty_like(x)
    code = L.pllgpu_dct2d_batch(int(kind), n0, n1, howmany, _dp(x), _dp(out))
    if code:
        raise _lib.PllGpuError(code, "dct2d_batch")
    return out
