"""The reference-side drop-in (include/fwi3d_we_op_gpu.hpp): the GPU
subclasses of nl_we_op_e / nl_we_op_vti / nl_we_op_a, compiled against the
reference's headers and driven through the reference's own
nl_we_op::forward / jacobianT calls (oracle/refside_driver.cpp), give the
unmodified operator's traces (1e-5) and gradient (1e-4)."""
import ctypes as C
import os

import numpy as np
import pytest

from fwi3d_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "librefside_gpu.so")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _lib():
    from oracle import refpy

    if not os.path.exists(LIB):
        pytest.skip("reference-side binding not built (make -C oracle)")
    lib = C.CDLL(LIB)
    fp, dp = C.POINTER(C.c_float), C.POINTER(C.c_double)
    lib.refside_run.argtypes = [C.POINTER(refpy.OracleParam), C.c_int, fp, fp, C.c_int, fp, C.c_int, fp, fp, dp, dp]
    lib.refside_run.restype = C.c_int
    return lib, refpy


def test_refside_library_exports():
    """Built (and linked against both libraries) wherever the reference is present; loads without a GPU."""
    lib, _ = _lib()
    assert hasattr(lib, "refside_run")


def _run(lib, refpy, sv, gpu, adj):
    op = refpy.make_param(sv)
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32).ctypes.data_as(C.POINTER(C.c_float))
    model = np.ascontiguousarray(sv.model, dtype=np.float32)
    w = np.ascontiguousarray(sv.wavelet, dtype=np.float32)
    s = np.ascontiguousarray(sv.par.sxyz[0], dtype=np.float32)
    r = np.ascontiguousarray(sv.par.rxyz[0], dtype=np.float32).reshape(-1, 5)
    nrc = refpy.nrcomp_of(sv)
    syn = np.zeros((nrc, r.shape[0], sv.nt_data), dtype=np.float64)
    grad = np.zeros(sv.model.shape, dtype=np.float64)
    a = np.ascontiguousarray(adj, dtype=np.float32) if adj is not None else None
    rc = lib.refside_run(C.byref(op), gpu, f(model), f(w), 1, f(s), r.shape[0], f(r),
                         a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None,
                         syn.ctypes.data_as(C.POINTER(C.c_double)), grad.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0
    return syn, grad


@pytest.mark.gpu
@pytest.mark.parametrize("physics", ["elastic", "vti", "acoustic"])
def test_gpu_subclass_through_reference_calls(physics):
    lib, refpy = _lib()
    if physics == "elastic":
        sv = synth.elastic_layered(n=26, nsteps=150, taper=6, rec_stride=3, nshots=1)
    elif physics == "vti":
        sv = synth.vti_layered(nx=26, ny=28, nz=24, nsteps=150, taper=6, rec_stride=3, nshots=1, dt=0.0005)
    else:
        sv = synth.acoustic_linear(n=28, nsteps=150, taper=6, rec_stride=3)
    n = sv.nx
    sv.par.sxyz = [[0.5 * n * sv.dx, 0.4 * sv.ny * sv.dx, 0.3 * sv.nz * sv.dx]]
    sv.par.sub = 1
    d_ref, _ = _run(lib, refpy, sv, 0, None)
    rng = np.random.default_rng(1)
    adj = (rng.standard_normal(d_ref.shape) * np.abs(d_ref).max()).astype(np.float32)
    d_ref, g_ref = _run(lib, refpy, sv, 0, adj)
    d_gpu, g_gpu = _run(lib, refpy, sv, 1, adj)
    e = rel(d_gpu, d_ref)
    eg = [rel(g_gpu[k], g_ref[k]) for k in range(min(3, sv.nmodels))]
    print(f"{physics}: traces {e:.3e}, gradient {eg}")
    assert e < 1e-5
    assert max(eg) < 1e-4
