"""ctypes binding of the in-tree ``libpllgpu.so`` (the ``pllgpu_`` C ABI of
``include/pllcart3d_gpu.h``).

There is no CPU fallback: if the library is missing or no CUDA device is
present, loading raises.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpllgpu.so")
DROPIN_PATH = os.path.join(HERE, "libpllcart3d_dropin.so")

_D = ctypes.c_double
_I = ctypes.c_int
_L = ctypes.c_long
_PD = ctypes.POINTER(ctypes.c_double)
_VP = ctypes.c_void_p

FIELD_NAMES = [
    "c_old", "c_new", "c_hn", "c_hnm1",
    "u_old", "u_new", "u_hn", "u_hnm1", "u_pg",
    "v_old", "v_new", "v_hn", "v_hnm1", "v_pg",
    "w_old", "w_new", "w_hn", "w_hnm1", "w_pg",
    "mu_old_cell", "mu_old_xy", "mu_old_xz", "mu_old_yz",
    "mu_new_cell", "mu_new_xy", "mu_new_xz", "mu_new_yz",
    "phi", "div",
]

ROUTINES = {
    "concentration": 0, "viscosity_new": 1, "xmom": 2, "ymom": 3, "zmom": 4,
    "velo_ghosts": 5, "divergence": 6, "phisolver": 7, "phi_ghosts": 8,
    "velo_correction": 9, "pressure_gradient": 10, "rotate": 11,
    "bulk_velo": 12, "find_cfl": 13, "substep": 14, "viscosity_exp": 15,
    "viscosity_nmvp": 16, "slope_parameter": 17,
}

ERRORS = {0: "ok", 1: "NaN or Inf in the velocity field", 2: "CUDA error",
          3: "device wait timed out", 4: "index out of bounds",
          5: "invalid argument", 6: "slope-parameter bisection did not converge"}


class Params(ctypes.Structure):
    """``pllgpu_params`` (include/pllcart3d_gpu.h)."""

    _fields_ = [
        ("nx", _I), ("ny", _I), ("nz", _I), ("nmvp", _I),
        ("X1", _D), ("X2", _D), ("Y1", _D), ("Y2", _D), ("Z1", _D), ("Z2", _D),
        ("Re", _D), ("Pe", _D), ("Vratio", _D), ("Fx", _D), ("Fy", _D),
        ("CFLmax", _D), ("Timestep", _D), ("Mum", _D), ("Lambda", _D),
        ("precision", _I), ("exact_dct", _I), ("use_graph", _I),
        ("dct_kernel", _I), ("explicit_kernel", _I), ("reserved", _I * 3),
    ]


class PllGpuError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"{what}: {ERRORS.get(code, code)} (code {code})")


_lib = None


def lib():
    """Load libpllgpu.so once (raises if absent: no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(
            f"{LIB_PATH} is not built; run `python -m pllcart3d_b200.build`")
    L = ctypes.CDLL(LIB_PATH, mode=os.RTLD_LOCAL)
    L.pllgpu_create.restype = _VP
    L.pllgpu_create.argtypes = [ctypes.POINTER(Params), _I]
    L.pllgpu_destroy.argtypes = [_VP]
    L.pllgpu_field_id.argtypes = [ctypes.c_char_p]
    L.pllgpu_dims.argtypes = [_VP, ctypes.POINTER(_I)]
    L.pllgpu_set_field.argtypes = [_VP, _I, _PD]
    L.pllgpu_get_field.argtypes = [_VP, _I, _PD]
    L.pllgpu_device_field.argtypes = [_VP, _I, ctypes.POINTER(_VP), ctypes.POINTER(_L), ctypes.POINTER(_L)]
    L.pllgpu_start.argtypes = [_VP]
    L.pllgpu_steps.argtypes = [_VP, _I]
    L.pllgpu_run_host.argtypes = [_VP, _I, _PD, _PD, _PD, _PD, _PD, _PD, _PD, _PD]
    L.pllgpu_routine.argtypes = [_VP, _I, _PD, _PD]
    L.pllgpu_sync.argtypes = [_VP]
    L.pllgpu_status.argtypes = [_VP]
    L.pllgpu_clear_status.argtypes = [_VP]
    L.pllgpu_last_dt.argtypes = [_VP]
    L.pllgpu_last_dt.restype = _D
    L.pllgpu_timestep.argtypes = [_VP]
    L.pllgpu_timestep.restype = _D
    L.pllgpu_tval.argtypes = [_VP]
    L.pllgpu_tval.restype = _D
    L.pllgpu_error_string.restype = ctypes.c_char_p
    L.pllgpu_kernels_per_step.argtypes = [_VP]
    L.pllgpu_stream.argtypes = [_VP]
    L.pllgpu_stream.restype = _VP
    L.pllgpu_profile_steps.argtypes = [_VP, _I, _I, ctypes.c_char_p, _PD,
                                       ctypes.POINTER(_I), ctypes.POINTER(_I)]
    L.pllgpu_tridiag_batch.argtypes = [_I, _I, _PD, _PD, _PD, _PD]
    L.pllgpu_dct2d_batch.argtypes = [_I, _I, _I, _I, _PD, _PD]
    L.pllgpu_diagnostics.argtypes = [_VP, _PD]
    L.pllgpu_set_timestep.argtypes = [_VP, _D]
    L.pllgpu_set_tval.argtypes = [_VP, _D]
    L.pllgpu_acoef.argtypes = [_VP, _I, _I, _PD]
    L.pllgpu_weno_batch.argtypes = [_I, _PD, _PD]
    L.pllgpu_tridiag_1rhs_batch.argtypes = [_I, _I, _PD, _PD, _PD, _PD]
    L.pllgpu_idct2d_batch.argtypes = [_I, _I, _I, _PD, _PD]
    L.pllgpu_dct2d_batch_noalloc.argtypes = [_I, _I, _I, _I, _VP, _VP, _VP]
    _S = ctypes.c_char_p
    L.pllgpu_resume.argtypes = [_VP, _D]
    L.pllgpu_write_snapshot.argtypes = [_VP, _I, _S]
    L.pllgpu_write_snapshot_ex.argtypes = [_VP, _I, _I, _S, _I]
    L.pllgpu_write_restart.argtypes = [_VP, _I, _I, _D, _D, _D, _D, _S]
    L.pllgpu_read_restart.argtypes = [_VP, _S, ctypes.POINTER(_I), ctypes.POINTER(_I), _PD, _PD]
    L.pllgpu_conc_average.argtypes = [_VP, _D, _S]
    L.pllgpu_find_wmax.argtypes = [_VP, _D, _S, _PD]
    L.pllgpu_find_max.argtypes = [_VP, _S, _PD, ctypes.POINTER(_I)]
    L.pllgpu_shift_conc.argtypes = [_VP, _D, _D, _I]
    _PI = ctypes.POINTER(_I)
    L.pllgpu_autotune.argtypes = [_VP, _I, _PI]
    L.pllgpu_tuning.argtypes = [_VP, _PI, _PI]
    L.pllgpu_set_tuning.argtypes = [_VP, _I, _I]
    L.pllgpu_ensemble_create.restype = _VP
    L.pllgpu_ensemble_create.argtypes = [_I, ctypes.POINTER(Params), _I]
    L.pllgpu_ensemble_destroy.argtypes = [_VP]
    L.pllgpu_ensemble_size.argtypes = [_VP]
    L.pllgpu_ensemble_member.restype = _VP
    L.pllgpu_ensemble_member.argtypes = [_VP, _I]
    L.pllgpu_ensemble_start.argtypes = [_VP]
    L.pllgpu_ensemble_steps.argtypes = [_VP, _I]
    L.pllgpu_ensemble_autotune.argtypes = [_VP, _I, _PI]
    L.pllgpu_ensemble_launches_per_step.argtypes = [_VP]
    L.pllgpu_ensemble_set_batching.argtypes = [_VP, _I]
    L.pllgpu_ensemble_classes.argtypes = [_VP]
    L.pllgpu_pack_cells.argtypes = [_VP, _VP]
    L.pllgpu_unpack_cells.argtypes = [_VP, _VP]
    L.pllgpu_copy_state.argtypes = [_VP, _VP]
    _lib = L
    return L


EXPORTED_SYMBOLS = [
    "pllgpu_create", "pllgpu_destroy", "pllgpu_field_id", "pllgpu_dims",
    "pllgpu_set_field", "pllgpu_get_field", "pllgpu_device_field",
    "pllgpu_start", "pllgpu_steps", "pllgpu_run_host", "pllgpu_routine",
    "pllgpu_sync", "pllgpu_status", "pllgpu_clear_status", "pllgpu_last_dt",
    "pllgpu_timestep", "pllgpu_tval", "pllgpu_error_string",
    "pllgpu_kernels_per_step", "pllgpu_tridiag_batch", "pllgpu_dct2d_batch",
    "pllgpu_stream", "pllgpu_profile_steps", "pllgpu_dct2d_batch_noalloc",
    "pllgpu_set_timestep", "pllgpu_set_tval", "pllgpu_acoef", "pllgpu_weno_batch",
    "pllgpu_tridiag_1rhs_batch", "pllgpu_idct2d_batch", "pllgpu_diagnostics",
    "pllgpu_resume", "pllgpu_write_snapshot", "pllgpu_write_snapshot_ex",
    "pllgpu_write_restart", "pllgpu_read_restart", "pllgpu_conc_average",
    "pllgpu_find_wmax", "pllgpu_find_max", "pllgpu_shift_conc",
    "pllgpu_autotune", "pllgpu_tuning", "pllgpu_set_tuning",
    "pllgpu_ensemble_create", "pllgpu_ensemble_destroy", "pllgpu_ensemble_size",
    "pllgpu_ensemble_member", "pllgpu_ensemble_start", "pllgpu_ensemble_steps",
    "pllgpu_ensemble_autotune", "pllgpu_ensemble_launches_per_step",
    "pllgpu_ensemble_set_batching", "pllgpu_ensemble_classes",
    "pllgpu_pack_cells", "pllgpu_unpack_cells", "pllgpu_copy_state",
]
