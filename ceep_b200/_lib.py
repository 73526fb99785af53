"""ctypes binding of include/ceep_b200.h (libceep_b200.so, built in-tree).

There is no fallback: if the shared library is missing or lacks a symbol,
importing the solvers raises.  ``build()`` compiles it with nvcc.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libceep_b200.so")

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64


class Desc2D(C.Structure):
    """Mirror of ``ceep2d_desc``."""
    _fields_ = [
        ("nx", I32), ("ny", I32), ("cpml", I32), ("ntx", I32), ("ntx_pad", I32),
        ("nprobe", I32), ("nsteps", I32), ("n_debye", I32), ("n_lorentz", I32),
        ("db", C.c_float), ("inv_dx", C.c_float), ("dt", C.c_float),
        ("ez", P * 2), ("hx", P * 2), ("hy", P * 2), ("psi_hy", P * 2), ("psi_hx", P * 2),
        ("psi_ezx", P * 2), ("psi_ezy", P * 2), ("j", P * 2), ("j_prev", P * 2),
        ("coef", P), ("ade_coef", P), ("cpml_b", P), ("cpml_c", P),
        ("src_xy", P), ("prb_xy", P), ("row_flags", P), ("waveform", P), ("probes", P),
        ("status", P), ("rows_per_block", I32),
    ]


class Desc3D(C.Structure):
    """Mirror of ``ceep3d_desc``."""
    _fields_ = [
        ("nx", I32), ("ny", I32), ("nz", I32), ("cpml", I32), ("ntx", I32), ("ntx_pad", I32),
        ("nprobe", I32), ("nsteps", I32), ("n_debye", I32), ("n_lorentz", I32),
        ("inv_dx", C.c_float), ("dt", C.c_float),
        ("ex", P), ("ey", P), ("ez", P), ("hx", P), ("hy", P), ("hz", P),
        ("psi_hxy", P), ("psi_hzy", P), ("psi_hyx", P), ("psi_hzx", P), ("psi_hxz", P), ("psi_hyz", P),
        ("j", P), ("j_prev", P), ("coef", P), ("ade_coef", P), ("cpml_b", P), ("cpml_c", P),
        ("src_xyz", P), ("prb_xyz", P), ("waveform", P), ("probes", P), ("z_rows", I32), ("shell_z_rows", I32),
    ]


# name -> (restype, argtypes)
_SIGS = {
    "ceep_version": (C.c_int, []),
    "ceep_last_error": (C.c_char_p, []),
    "ceep2d_plan_create": (C.c_int, [C.POINTER(Desc2D), C.POINTER(P)]),
    "ceep2d_plan_run": (C.c_int, [P, I64, I64, P, C.c_int]),
    "ceep2d_plan_destroy": (C.c_int, [P]),
    "ceep2d_launches_per_step": (C.c_int, [P]),
    "ceep2d_plan_set_temporal_block": (C.c_int, [P, C.c_int]),
    "ceep2d_plan_set_frame_split": (C.c_int, [P, I32]),
    "ceep2d_material_coefficients": (C.c_int, [P, P, P, I32, I32, I32, I32, C.c_double, C.c_double, P, P, P]),
    "ceep2d_plan_temporal_block": (C.c_int, [P]),
    "ceep2d_plan_launches": (I64, [P, I64]),
    "ceep2d_plan_set_sentinel": (C.c_int, [P, I32]),
    "ceep2d_plan_set_wait_limit": (C.c_int, [P, C.c_uint64]),
    "ceep2d_plan_inject_copy_fault": (C.c_int, [P, I32]),
    "ceep2d_plan_current_buffer": (C.c_int, [P]),
    "ceep2d_plan_reset": (C.c_int, [P]),
    "ceep2d_desc_size": (I64, []),
    "ceep2d_plan_rows": (C.c_int, [P]),
    "ceep2d_plan_run_save": (C.c_int, [P, I64, I64, P, C.c_int, P, P, I64]),
    "ceep2d_plan_set_current_buffer": (C.c_int, [P, C.c_int]),
    "ceep2d_adjoint_create": (C.c_int, [P, P, C.POINTER(P)]),
    "ceep2d_adjoint_run": (C.c_int, [P, I64, I64, P, P, I64, P]),
    "ceep2d_adjoint_reset": (C.c_int, [P]),
    "ceep2d_adjoint_destroy": (C.c_int, [P]),
    "ceep2d_adjoint_desc_size": (I64, []),
    "ceep2d_adjoint_rows": (C.c_int, [P]),
    "ceep2d_adjoint_set_rows": (C.c_int, [P, I32]),
    "ceep2d_pack_workspace_bytes": (I64, [C.POINTER(P), I32]),
    "ceep2d_pack_create": (C.c_int, [C.POINTER(P), I32, P, I64, P, C.POINTER(P)]),
    "ceep2d_pack_run": (C.c_int, [P, I64, I64, P, C.c_int]),
    "ceep2d_pack_tiles": (C.c_int, [P, I32]),
    "ceep2d_pack_set_temporal_block": (C.c_int, [P, C.c_int]),
    "ceep2d_pack_temporal_block": (C.c_int, [P]),
    "ceep2d_pack_set_packing": (C.c_int, [P, C.c_int]),
    "ceep2d_pack_packing": (C.c_int, [P]),
    "ceep2d_pack_destroy": (C.c_int, [P]),
    "ceep3d_plan_create": (C.c_int, [C.POINTER(Desc3D), C.POINTER(P)]),
    "ceep3d_plan_run": (C.c_int, [P, I64, I64, P, C.c_int]),
    "ceep3d_plan_destroy": (C.c_int, [P]),
    "ceep3d_desc_size": (I64, []),
    "ceep3d_plan_run_save": (C.c_int, [P, I64, I64, P, C.c_int, P, I64, C.c_int]),
    "ceep2s_plan_create": (C.c_int, [P, C.POINTER(P)]),
    "ceep2s_plan_run": (C.c_int, [P, I64, I64, P, C.c_int]),
    "ceep2s_plan_destroy": (C.c_int, [P]),
    "ceep2s_plan_current_buffer": (C.c_int, [P]),
    "ceep2s_plan_set_current_buffer": (C.c_int, [P, C.c_int]),
    "ceep2s_desc_size": (I64, []),
    "ceep3d_adjoint_create": (C.c_int, [P, P, C.POINTER(P)]),
    "ceep3d_adjoint_run": (C.c_int, [P, I64, I64, P, I64, P]),
    "ceep3d_adjoint_grad_slots": (I32, [P]),
    "ceep3d_adjoint_destroy": (C.c_int, [P]),
    "ceep3d_adjoint_desc_size": (I64, []),
    "ceep_dft": (C.c_int, [P, P, P, I32, I32, I32, I32, P]),
    "ceep_das_workspace_bytes": (I64, [I32, I32, I32]),
    "ceep_das": (C.c_int, [P, P, P, I32, I32, I32, I32, C.c_float, C.c_float, C.c_float, C.c_int, P, P, P]),
    "ceep_das_time": (C.c_int, [P, P, I32, I32, I32, C.c_double, C.c_double, P, P]),
    "ceep_dmas_workspace_bytes": (I64, [I32, I32]),
    "ceep_brain_phantom_2d": (C.c_int, [I32, I32, I32, C.c_double, P, P, P, P, P, P, P]),
    "ceep_dmas": (C.c_int, [P, P, P, I32, I32, I32, I32, C.c_float, C.c_float, C.c_float, C.c_int, P, P, P]),
    "ceep_das_noalloc_capacity": (I64, []),
    "ceep_das_noalloc": (C.c_int, [P, P, P, I32, I32, I32, I32, C.c_float, C.c_float, C.c_float, C.c_int, P, P]),
}

_lib = None


class CeepError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib().ceep_last_error().decode(errors="replace")
        super().__init__(f"{where} failed (status {code}): {msg}")
        self.code = code


def lib():
    """Load libceep_b200.so once; raise if it is absent or incomplete."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m ceep_b200.csrc.build`")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        if h.ceep2d_desc_size() != C.sizeof(Desc2D) or h.ceep3d_desc_size() != C.sizeof(Desc3D):
            raise ImportError("descriptor layout mismatch between header and binding")
        _lib = h
    return _lib


def check(code: int, where: str) -> None:
    if code != 0:
        raise CeepError(code, where)


def exported_symbols():
    return list(_SIGS)
