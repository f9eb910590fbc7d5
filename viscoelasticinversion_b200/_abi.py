"""ctypes mirror of include/visco_b200.h and the loader of libvisco_b200.so.

The library is the only compute path: if it is missing, every entry point
raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libvisco_b200.so"

VI_HALF = 4
VI_MAX_SLS = 5

VI_OK = 0
VI_ERR_ARG = 1
VI_ERR_CFL = 2
VI_ERR_BUDGET = 3
VI_ERR_TIMEOUT = 4
VI_ERR_CUDA = 5
VI_ERR_NONFINITE = 6
VI_ERR_STATE = 7

VI_MEDIUM_ISO = 0
VI_MEDIUM_VTI = 1
VI_MEDIUM_TTI = 2
VI_F32 = 0
VI_F64 = 1
VI_F32C = 2  # FP32 fields, split-pair stress update compensated (residues in the plan)
PRECISIONS = {"f32": VI_F32, "f64": VI_F64, "f32c": VI_F32C}
VI_SRC_EXPLOSIVE = 0
VI_SRC_FORCE_X = 1
VI_SRC_FORCE_Z = 2

MEDIUM_KINDS = {"iso": VI_MEDIUM_ISO, "vti": VI_MEDIUM_VTI, "tti": VI_MEDIUM_TTI}


class ViConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("nz", C.c_int32),
        ("dx", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
        ("medium", C.c_int32), ("precision", C.c_int32), ("nsls", C.c_int32),
        ("free_surface", C.c_int32),
        ("tau_sls", C.c_double * VI_MAX_SLS),
        ("pml_thickness", C.c_int32),
        ("pml_left", C.c_int32), ("pml_right", C.c_int32),
        ("pml_top", C.c_int32), ("pml_bottom", C.c_int32),
        ("pml_d0", C.c_double), ("pml_vmax", C.c_double),
        ("pml_reflection", C.c_double), ("pml_power", C.c_double),
        ("pml_alpha_max", C.c_double), ("pml_kappa_max", C.c_double),
    ]


class ViMedium(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("rho", "c11", "c13", "c15", "c33", "c35", "c55", "tau")]


class ViFields(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("vx", "vz", "sxx", "szz", "sxz", "m")] + [
        ("m_plane_stride", C.c_int64)]


class ViSource(C.Structure):
    _fields_ = [("i", C.c_int32), ("j", C.c_int32), ("kind", C.c_int32),
                ("pad_", C.c_int32), ("amp", C.c_double)]


class ViReceiver(C.Structure):
    _fields_ = [("i", C.c_int32), ("j", C.c_int32)]


class ViShot(C.Structure):
    _fields_ = [
        ("nsrc", C.c_int32), ("src_host", C.POINTER(ViSource)),
        ("wavelet_dev", C.c_void_p), ("wavelet_nt", C.c_int32),
        ("nrec", C.c_int32), ("rec_host", C.POINTER(ViReceiver)),
        ("traces_dev", C.c_void_p), ("traces_nt", C.c_int32),
    ]


class ViServeConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("slice_steps", C.c_int32), ("max_active", C.c_int32),
                ("policy", C.c_int32), ("hbm_budget_bytes", C.c_int64), ("lanes", C.c_int32),
                ("pad_", C.c_int32)]


class ViRequest(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("nt", C.c_int32), ("cfg", ViConfig), ("medium_host", ViMedium),
        ("nsrc", C.c_int32), ("wavelet_nt", C.c_int32), ("src_host", C.POINTER(ViSource)),
        ("wavelet_host", C.c_void_p), ("nrec", C.c_int32), ("pad_", C.c_int32),
        ("rec_host", C.POINTER(ViReceiver)), ("traces_host", C.c_void_p), ("obs_host", C.c_void_p),
        ("grad_host", C.c_void_p), ("misfit_host", C.c_void_p),
    ]


VI_SERVE_SHORTEST_FIRST, VI_SERVE_ROUND_ROBIN = 0, 1
VI_REQ_FORWARD, VI_REQ_GRADIENT = 0, 1
VI_REQ_QUEUED, VI_REQ_RUNNING, VI_REQ_DONE, VI_REQ_FAILED = 0, 1, 2, 3


class ViError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class CFLError(ViError):
    pass


class BudgetError(ViError):
    pass


_lib = None

# (name, restype, argtypes) of every exported entry point
_SIGNATURES = [
    ("vi_version", C.c_int, []),
    ("vi_last_error", C.c_char_p, []),
    ("vi_plan_create", C.c_int, [C.POINTER(ViConfig), C.POINTER(C.c_void_p)]),
    ("vi_plan_destroy", C.c_int, [C.c_void_p]),
    ("vi_plan_reset", C.c_int, [C.c_void_p, C.c_void_p]),
    ("vi_plan_workspace_bytes", C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    ("vi_plan_status", C.c_int, [C.c_void_p, C.c_void_p]),
    ("vi_plan_last_kernel", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("vi_plan_set_wave", C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    ("vi_step", C.c_int, [C.c_void_p, C.POINTER(ViMedium), C.POINTER(ViFields),
                          C.POINTER(ViShot), C.c_int32, C.c_int32, C.c_int32, C.c_void_p]),
    ("vi_step_noalloc", C.c_int, [C.c_void_p, C.POINTER(ViMedium), C.POINTER(ViFields),
                                  C.POINTER(ViShot), C.c_int32, C.c_int32, C.c_void_p]),
    ("vi_forward_host", C.c_int, [C.c_void_p, C.POINTER(ViMedium), C.c_int32,
                                  C.POINTER(ViSource), C.c_void_p, C.c_int32,
                                  C.POINTER(ViReceiver), C.c_int32, C.c_void_p,
                                  C.POINTER(ViFields)]),
    ("vi_diff", C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                          C.c_int32, C.c_double, C.c_void_p]),
    ("vi_batch_create", C.c_int, [C.POINTER(ViConfig), C.c_int32, C.POINTER(C.c_void_p)]),
    ("vi_batch_destroy", C.c_int, [C.c_void_p]),
    ("vi_batch_set_shot", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(ViMedium),
                                    C.POINTER(ViFields), C.POINTER(ViShot), C.c_int32]),
    ("vi_batch_run", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    ("vi_batch_status", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]),
    ("vi_serve_start", C.c_int, [C.POINTER(ViServeConfig), C.POINTER(C.c_void_p)]),
    ("vi_serve_submit", C.c_int, [C.c_void_p, C.POINTER(ViRequest), C.POINTER(C.c_uint64)]),
    ("vi_serve_poll", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    ("vi_serve_wait", C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.POINTER(C.c_int32)]),
    ("vi_serve_stop", C.c_int, [C.c_void_p]),
    ("vi_gradient", C.c_int, [C.c_void_p, C.POINTER(ViMedium), C.POINTER(ViShot), C.c_int32,
                              C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                              C.POINTER(C.c_double), C.c_void_p]),
    ("vi_gradient_velocity", C.c_int, [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                       C.c_void_p, C.c_void_p]),
    ("vi_gradient_thomsen", C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p]),
    ("vi_gradient_tti", C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                  C.c_void_p]),
    ("vi_medium_from_velocity", C.c_int, [C.c_int32, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_double, C.POINTER(ViMedium), C.c_void_p]),
]

VI_BATCH_NO_GRAPH = 1
VI_BATCH_RETUNE = 2


def exported_names() -> list[str]:
    return [s[0] for s in _SIGNATURES]


def lib():
    """Loads libvisco_b200.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is not built; run `python -m viscoelasticinversion_b200.build` "
                "(there is no CPU fallback)")
        handle = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | getattr(os, "RTLD_LOCAL", 0))
        for name, res, args in _SIGNATURES:
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(rc: int) -> None:
    if rc == VI_OK:
        return
    msg = lib().vi_last_error().decode(errors="replace")
    cls = CFLError if rc == VI_ERR_CFL else BudgetError if rc == VI_ERR_BUDGET else ViError
    raise cls(rc, msg)
