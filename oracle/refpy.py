"""ctypes binding of the CPU oracle built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use this module as the checker; the product never imports it.

The libraries are the reference's own sources (nmbader/fwi3d src/cpp/*.cpp)
compiled unmodified, driven by oracle/ref_driver.cpp exactly as
src/main/we_modeling.cpp:72-90 (modeling) and src/cpp/optimization.cpp:41-50,181
(forward then adjoint on the same per-shot operator) drive them.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "_ref")


class OracleParam(C.Structure):
    _fields_ = [
        ("nmodels", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("ox", C.c_float), ("oy", C.c_float), ("oz", C.c_float),
        ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
        ("nt_data", C.c_int), ("dt_data", C.c_float),
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
        ("soft_clip", C.c_int), ("verbose", C.c_int), ("nthreads", C.c_int),
    ]


class OracleInfo(C.Structure):
    _fields_ = [("dt", C.c_double), ("nt", C.c_int), ("sub", C.c_int), ("courant", C.c_double),
                ("nscomp", C.c_int), ("nrcomp", C.c_int)]


_libs = {}


def lib_path(precision: str) -> str:
    return os.path.join(LIBDIR, f"libfwi3d_ref_{precision}.so")


def available(precision: str = "fp32") -> bool:
    return os.path.exists(lib_path(precision))


def _lib(precision: str):
    if precision not in _libs:
        path = lib_path(precision)
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library {path} is not built (make -C oracle)")
        lib = C.CDLL(path)
        fp = C.POINTER(C.c_float)
        dp = C.POINTER(C.c_double)
        lib.oracle_modeling.argtypes = [C.POINTER(OracleParam), fp, fp, C.c_int, fp, C.c_int, fp, dp,
                                        C.POINTER(OracleInfo)]
        lib.oracle_modeling.restype = C.c_int
        lib.oracle_forward_jacobianT.argtypes = [C.POINTER(OracleParam), fp, fp, C.c_int, fp, C.c_int, fp,
                                                 fp, dp, dp, C.POINTER(OracleInfo)]
        lib.oracle_forward_jacobianT.restype = C.c_int
        lib.oracle_data_t_size.restype = C.c_int
        _libs[precision] = lib
    return _libs[precision]


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_param(sv, nthreads: int = 0) -> OracleParam:
    p = sv.par
    op = OracleParam()
    op.nmodels = sv.nmodels
    op.nx, op.ny, op.nz = sv.nx, sv.ny, sv.nz
    op.ox, op.oy, op.oz = sv.ox, sv.oy, sv.oz
    op.dx, op.dy, op.dz = sv.dx, sv.dy, sv.dz
    op.nt_data, op.dt_data = sv.nt_data, sv.dt_data
    op.courant, op.dt, op.sub = p.courant, p.dt, p.sub
    op.resampling_linear = 1 if p.resampling == "linear" else 0
    op.sinc_half_length = p.sinc_half_length
    op.mt = int(p.mt)
    op.fangle, op.fazimuth = p.fangle, p.fazimuth
    op.mxx, op.myy, op.mzz, op.mxy, op.mxz, op.myz = p.mxx, p.myy, p.mzz, p.mxy, p.mxz, p.myz
    op.seismotype, op.gl = p.seismotype, p.gl
    for i, v in enumerate(p.bc):
        op.bc[i] = v
    for i, v in enumerate(p.taper):
        op.taper[i] = v
    op.free_surface_stiffness, op.taper_strength = p.free_surface_stiffness, p.taper_strength
    op.vpmin, op.vpmax, op.vsmin, op.vsmax = p.vpmin, p.vpmax, p.vsmin, p.vsmax
    op.rhomin, op.rhomax = p.rhomin, p.rhomax
    op.deltamin, op.deltamax, op.epsilonmin, op.epsilonmax = p.deltamin, p.deltamax, p.epsilonmin, p.epsilonmax
    op.gammamin, op.gammamax = p.gammamin, p.gammamax
    op.soft_clip, op.verbose, op.nthreads = int(p.soft_clip), p.verbose, nthreads
    return op


def nrcomp_of(sv) -> int:
    if sv.nmodels == 2:
        return 1
    return 1 if sv.par.gl > 0 else 3


def modeling(sv, shot: int = 0, precision: str = "fp32", nthreads: int = 0):
    """Reference traces [nrcomp][nr][nt_data] (float64) for one shot, plus info."""
    lib = _lib(precision)
    op = make_param(sv, nthreads)
    model = np.ascontiguousarray(sv.model, dtype=np.float32)
    w = np.ascontiguousarray(sv.wavelet, dtype=np.float32)
    ncomp = 1 if w.ndim == 1 else w.shape[0]
    s = np.ascontiguousarray(sv.par.sxyz[shot], dtype=np.float32)
    r = np.ascontiguousarray(sv.par.rxyz[shot], dtype=np.float32).reshape(-1, 5)
    nr = r.shape[0]
    out = np.zeros((nrcomp_of(sv), nr, sv.nt_data), dtype=np.float64)
    info = OracleInfo()
    rc = lib.oracle_modeling(C.byref(op), _fptr(model), _fptr(w), ncomp, _fptr(s), nr, _fptr(r), _dptr(out),
                             C.byref(info))
    if rc != 0:
        raise RuntimeError(f"oracle_modeling failed ({rc})")
    return out, info


def forward_jacobianT(sv, adj_data: np.ndarray, shot: int = 0, precision: str = "fp32", nthreads: int = 0):
    """Forward traces and the adjoint-state gradient (apply_jacobianT, add=false)
    for one shot; ``adj_data`` has the data shape [nrcomp][nr][nt_data]."""
    lib = _lib(precision)
    op = make_param(sv, nthreads)
    model = np.ascontiguousarray(sv.model, dtype=np.float32)
    w = np.ascontiguousarray(sv.wavelet, dtype=np.float32)
    ncomp = 1 if w.ndim == 1 else w.shape[0]
    s = np.ascontiguousarray(sv.par.sxyz[shot], dtype=np.float32)
    r = np.ascontiguousarray(sv.par.rxyz[shot], dtype=np.float32).reshape(-1, 5)
    nr = r.shape[0]
    a = np.ascontiguousarray(adj_data, dtype=np.float32)
    syn = np.zeros((nrcomp_of(sv), nr, sv.nt_data), dtype=np.float64)
    nm = min(3, sv.nmodels)
    grad = np.zeros((nm, sv.ny, sv.nx, sv.nz), dtype=np.float64)
    info = OracleInfo()
    rc = lib.oracle_forward_jacobianT(C.byref(op), _fptr(model), _fptr(w), ncomp, _fptr(s), nr, _fptr(r),
                                      _fptr(a), _dptr(syn), _dptr(grad), C.byref(info))
    if rc != 0:
        raise RuntimeError(f"oracle_forward_jacobianT failed ({rc})")
    return syn, grad, info


class OracleSolver(C.Structure):
    _fields_ = [("solver", C.c_int), ("lsearch", C.c_int), ("niter", C.c_int), ("max_trial", C.c_int),
                ("threshold", C.c_float), ("ls_c1", C.c_float), ("ls_c2", C.c_float), ("ls_a0", C.c_float),
                ("ls_a1", C.c_float), ("ls_max_step", C.c_float), ("ls_version", C.c_int), ("lbfgs_m", C.c_int),
                ("nlcg_method", C.c_int), ("normalize_obj_func", C.c_int)]


SOLVERS = {"none": 0, "lbfgs": 1, "nlcg": 2, "nlsd": 3}
LSEARCH = {"weak_wolfe": 0, "regular_wolfe": 1}


def fwi(sv, observed: np.ndarray, solver: str = "none", lsearch: str = "regular_wolfe", niter: int = 1,
        max_trial: int = 10, normalize: bool = True, precision: str = "fp32", nthreads: int = 0, lbfgs_m: int = 5,
        nlcg_method: int = 0, c1: float = 1e-4, c2: float = 0.9, a0: float = 1.0, a1: float = 0.0):
    """The reference's FWI objective (nlls_fwi, optimization.cpp) on all shots
    of the survey, or a run of its solver (nlsolver.cpp) from sv.model.
    Returns dict(f=[objective history], model=final model, grad=gradient at
    the last evaluated model, feval, geval)."""
    lib = _lib(precision)
    if not hasattr(lib, "_fwi_bound"):
        fp = C.POINTER(C.c_float)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        lib.oracle_fwi.argtypes = [C.POINTER(OracleParam), fp, fp, C.c_int, C.c_int, fp, C.c_int, fp, fp,
                                   C.POINTER(OracleSolver), dp, ip, dp, dp, ip]
        lib.oracle_fwi.restype = C.c_int
        lib._fwi_bound = True
    op = make_param(sv, nthreads)
    model = np.ascontiguousarray(sv.model, dtype=np.float32)
    w = np.ascontiguousarray(sv.wavelet, dtype=np.float32)
    ncomp = 1 if w.ndim == 1 else w.shape[0]
    ns = len(sv.par.sxyz)
    s = np.ascontiguousarray(np.asarray(sv.par.sxyz, dtype=np.float32)[:, :3])
    nr = len(sv.par.rxyz[0])
    r = np.ascontiguousarray(np.asarray(sv.par.rxyz, dtype=np.float32).reshape(ns, nr, 5))
    obs = np.ascontiguousarray(observed, dtype=np.float32)
    so = OracleSolver(SOLVERS[solver], LSEARCH[lsearch], niter, max_trial, 0.0, c1, c2, a0, a1, 1e6, 0, lbfgs_m,
                      nlcg_method, 1 if normalize else 0)
    fh = np.zeros(niter + 2, dtype=np.float64)
    nf = C.c_int()
    mo = np.zeros(model.shape, dtype=np.float64)
    go = np.zeros(model.shape, dtype=np.float64)
    counts = (C.c_int * 2)()
    rc = lib.oracle_fwi(C.byref(op), _fptr(model), _fptr(w), ncomp, ns, _fptr(s), nr, _fptr(r), _fptr(obs),
                        C.byref(so), _dptr(fh), C.byref(nf), _dptr(mo), _dptr(go), counts)
    if rc != 0:
        raise RuntimeError(f"oracle_fwi failed ({rc})")
    return {"f": fh[: nf.value].tolist(), "model": mo, "grad": go, "feval": counts[0], "geval": counts[1]}
