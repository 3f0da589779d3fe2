"""ctypes binding of libfwi3d_b200.so (the C ABI of include/fwi3d_gpu.h).

The library is built in-tree (fwi3d_b200/build.py).  There is no CPU fallback:
if the library is missing the import of the operators raises, and every call
that needs a GPU returns FWI_ERR_NOGPU, raised here as FwiError.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
# FWI3D_B200_LIB points at another build of the library (e.g. an instrumented one)
LIB_PATH = os.environ.get("FWI3D_B200_LIB") or os.path.join(HERE, "libfwi3d_b200.so")

FWI_OK = 0
FWI_ERR_ARG = -1
FWI_ERR_OOM = -2
FWI_ERR_CUDA = -3
FWI_ERR_NAN = -4
FWI_ERR_STATE = -5
FWI_ERR_UNSUPPORTED = -6
FWI_ERR_NOGPU = -7

# Every entry point declared in include/fwi3d_gpu.h.
EXPORTS = [
    "fwi_param_default", "fwi_op_create", "fwi_op_forward", "fwi_op_jacobianT", "fwi_op_get_info",
    "fwi_op_destroy", "fwi_forward_batch", "fwi_batch_create", "fwi_batch_reset", "fwi_batch_run",
    "fwi_batch_sync", "fwi_batch_stream", "fwi_batch_traces", "fwi_batch_get_info", "fwi_batch_destroy",
    "fwi_last_error", "fwi_version", "fwi_elastic_step_static", "fwi_batch_time_main_kernel",
    "fwi_batch_main_kernel_time", "fwi_objective_create", "fwi_objective_evaluate", "fwi_objective_device_bytes",
    "fwi_objective_destroy", "fwi_batch_enable_slots", "fwi_batch_ready", "fwi_batch_join", "fwi_batch_release",
    "fwi_batch_slot_time", "fwi_batch_slot_traces", "fwi_objective_evaluate_shots", "fwi_objective_set_shots",
]


class FwiError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("ox", C.c_float), ("oy", C.c_float), ("oz", C.c_float),
                ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float)]


class CParam(C.Structure):
    _fields_ = [
        ("courant", C.c_float), ("dt", C.c_float), ("sub", C.c_int),
        ("resampling_linear", C.c_int), ("sinc_half_length", C.c_int),
        ("mt", C.c_int), ("fangle", C.c_float), ("fazimuth", C.c_float),
        ("mxx", C.c_float), ("myy", C.c_float), ("mzz", C.c_float),
        ("mxy", C.c_float), ("mxz", C.c_float), ("myz", C.c_float),
        ("seismotype", C.c_int), ("gl", C.c_float),
        ("bc", C.c_int * 6), ("taper", C.c_int * 6),
        ("free_surface_stiffness", C.c_float), ("taper_strength", C.c_float),
        ("vpmin", C.c_float), ("vpmax", C.c_float), ("vsmin", C.c_float), ("vsmax", C.c_float),
        ("rhomin", C.c_float), ("rhomax", C.c_float),
        ("deltamin", C.c_float), ("deltamax", C.c_float), ("epsilonmin", C.c_float),
        ("epsilonmax", C.c_float), ("gammamin", C.c_float), ("gammamax", C.c_float),
        ("soft_clip", C.c_int), ("verbose", C.c_int), ("snapshot_storage", C.c_int),
        ("snapshot_budget_gb", C.c_float), ("checkpoint_slots", C.c_int), ("checkpoint_precision", C.c_int),
    ]


class OpInfo(C.Structure):
    _fields_ = [("dt", C.c_float), ("nt", C.c_int), ("sub", C.c_int), ("nscomp", C.c_int),
                ("nrcomp", C.c_int), ("nr", C.c_int), ("device_bytes", C.c_int64)]


_lib: Optional[C.CDLL] = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -m fwi3d_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(LIB_PATH)
    fp = C.POINTER(C.c_float)
    vp = C.c_void_p
    lib.fwi_param_default.argtypes = [C.POINTER(CParam)]
    lib.fwi_param_default.restype = None
    lib.fwi_op_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(Grid), C.c_int, C.POINTER(CParam), fp, C.c_int,
                                  C.c_int, C.c_float, fp, C.c_int, fp]
    lib.fwi_op_create.restype = C.c_int
    lib.fwi_op_forward.argtypes = [vp, C.c_int, fp, fp]
    lib.fwi_op_forward.restype = C.c_int
    lib.fwi_op_jacobianT.argtypes = [vp, C.c_int, fp, fp, fp]
    lib.fwi_op_jacobianT.restype = C.c_int
    lib.fwi_op_get_info.argtypes = [vp, C.POINTER(OpInfo)]
    lib.fwi_op_get_info.restype = C.c_int
    lib.fwi_op_destroy.argtypes = [vp]
    lib.fwi_op_destroy.restype = None
    lib.fwi_forward_batch.argtypes = [C.c_int, C.POINTER(Grid), C.c_int, C.POINTER(CParam), fp, fp, C.c_int, C.c_int,
                                      C.c_float, C.c_int, fp, C.c_int, fp, fp]
    lib.fwi_forward_batch.restype = C.c_int
    lib.fwi_batch_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(Grid), C.c_int, C.POINTER(CParam), fp, fp,
                                     C.c_int, C.c_int, C.c_float, C.c_int, fp, C.c_int, fp]
    lib.fwi_batch_create.restype = C.c_int
    for name in ("fwi_batch_reset", "fwi_batch_sync"):
        getattr(lib, name).argtypes = [vp]
        getattr(lib, name).restype = C.c_int
    lib.fwi_batch_run.argtypes = [vp, C.c_int]
    lib.fwi_batch_run.restype = C.c_int
    lib.fwi_batch_stream.argtypes = [vp, C.POINTER(vp)]
    lib.fwi_batch_stream.restype = C.c_int
    lib.fwi_batch_traces.argtypes = [vp, fp]
    lib.fwi_batch_traces.restype = C.c_int
    lib.fwi_batch_ready.argtypes = [vp, C.POINTER(C.c_int)]
    lib.fwi_batch_ready.restype = C.c_int
    lib.fwi_batch_enable_slots.argtypes = [vp]
    lib.fwi_batch_enable_slots.restype = C.c_int
    lib.fwi_batch_join.argtypes = [vp, C.c_int, fp, fp]
    lib.fwi_batch_join.restype = C.c_int
    lib.fwi_batch_release.argtypes = [vp, C.c_int]
    lib.fwi_batch_release.restype = C.c_int
    lib.fwi_batch_slot_time.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.fwi_batch_slot_time.restype = C.c_int
    lib.fwi_batch_slot_traces.argtypes = [vp, C.c_int, fp]
    lib.fwi_batch_slot_traces.restype = C.c_int
    lib.fwi_objective_evaluate_shots.argtypes = [vp, fp, C.POINTER(C.c_double), fp]
    lib.fwi_objective_evaluate_shots.restype = C.c_int
    lib.fwi_objective_set_shots.argtypes = [vp, fp, fp, fp]
    lib.fwi_objective_set_shots.restype = C.c_int
    lib.fwi_batch_get_info.argtypes = [vp, C.POINTER(OpInfo), C.POINTER(C.c_int)]
    lib.fwi_batch_get_info.restype = C.c_int
    lib.fwi_batch_destroy.argtypes = [vp]
    lib.fwi_batch_destroy.restype = None
    lib.fwi_elastic_step_static.argtypes = [C.POINTER(Grid), C.c_int, C.POINTER(C.c_int), C.c_float, vp, vp, vp,
                                            vp, vp]
    lib.fwi_elastic_step_static.restype = C.c_int
    lib.fwi_batch_time_main_kernel.argtypes = [vp, C.c_int]
    lib.fwi_batch_time_main_kernel.restype = C.c_int
    lib.fwi_batch_main_kernel_time.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int64),
                                               C.POINTER(C.c_char_p)]
    lib.fwi_batch_main_kernel_time.restype = C.c_int
    lib.fwi_objective_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(Grid), C.c_int, C.POINTER(CParam), fp,
                                         C.c_int, C.c_int, C.c_float, C.c_int, fp, C.c_int, fp, fp, C.c_int, C.c_int]
    lib.fwi_objective_create.restype = C.c_int
    lib.fwi_objective_evaluate.argtypes = [vp, fp, C.POINTER(C.c_double), fp, fp]
    lib.fwi_objective_evaluate.restype = C.c_int
    lib.fwi_objective_device_bytes.argtypes = [vp]
    lib.fwi_objective_device_bytes.restype = C.c_int64
    lib.fwi_objective_destroy.argtypes = [vp]
    lib.fwi_objective_destroy.restype = None
    lib.fwi_last_error.restype = C.c_char_p
    lib.fwi_version.restype = C.c_char_p
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != FWI_OK:
        msg = load().fwi_last_error().decode(errors="replace")
        raise FwiError(rc, msg)


def fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))
