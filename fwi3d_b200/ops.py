"""Wave-equation operators with the reference's interface, running on the GPU.

Mirrors nmbader/fwi3d ``src/include/we_op.hpp``:

============================  ===========================================
reference (C++)               here (Python over the C ABI)
============================  ===========================================
nl_we_op_e(domain, allsrc,    nl_we_op_e(domain, allsrc, s, par, dt_data)
           s, par)
nl_we_op_vti, nl_we_op_a      nl_we_op_vti, nl_we_op_a
forward(add, mod, dat)        forward(add, mod, dat) -> dat
jacobianT(add, mod, mod0,     jacobianT(add, mod, mod0, dat) -> mod
          dat)
apply_forward / apply_        same, on raw float32 arrays
jacobianT
_par, _src, _allsrc           _par, _src, _allsrc
getDomain() / getRange()      domain_shape / range_shape
============================  ===========================================

Arrays are numpy float32 in the reference layouts: model [nmodels][ny][nx][nz],
data [nrcomp][nr][nt_data], wavelet [nt] (duplicated as analyzeWavelet does)
or [ns][ncomp][nt] (one entry per shot).  A failing call raises FwiError
carrying the C status, where the reference would exit(123).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import ctypes as C
import numpy as np

from . import _lib
from .param import Param


@dataclass
class Domain:
    """Model hypercube: axes Z (fast), X, Y and the parameter axis."""

    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    nmodels: int
    ox: float = 0.0
    oy: float = 0.0
    oz: float = 0.0

    @property
    def shape(self):
        return (self.nmodels, self.ny, self.nx, self.nz)

    def grid(self) -> _lib.Grid:
        return _lib.Grid(self.nx, self.ny, self.nz, self.ox, self.oy, self.oz, self.dx, self.dy, self.dz)


def to_cparam(p: Param) -> _lib.CParam:
    lib = _lib.load()
    c = _lib.CParam()
    lib.fwi_param_default(C.byref(c))
    c.courant, c.dt, c.sub = p.courant, p.dt, p.sub
    c.resampling_linear = 1 if p.resampling == "linear" else 0
    c.sinc_half_length = p.sinc_half_length
    c.mt = int(bool(p.mt))
    c.fangle, c.fazimuth = p.fangle, p.fazimuth
    c.mxx, c.myy, c.mzz, c.mxy, c.mxz, c.myz = p.mxx, p.myy, p.mzz, p.mxy, p.mxz, p.myz
    c.seismotype, c.gl = p.seismotype, p.gl
    for i, v in enumerate(p.bc):
        c.bc[i] = int(v)
    for i, v in enumerate(p.taper):
        c.taper[i] = int(v)
    c.free_surface_stiffness, c.taper_strength = p.free_surface_stiffness, p.taper_strength
    c.vpmin, c.vpmax, c.vsmin, c.vsmax, c.rhomin, c.rhomax = p.vpmin, p.vpmax, p.vsmin, p.vsmax, p.rhomin, p.rhomax
    c.deltamin, c.deltamax = p.deltamin, p.deltamax
    c.epsilonmin, c.epsilonmax = p.epsilonmin, p.epsilonmax
    c.gammamin, c.gammamax = p.gammamin, p.gammamax
    c.soft_clip, c.verbose = int(bool(p.soft_clip)), p.verbose
    c.snapshot_storage = int(getattr(p, "snapshot_storage", 0))
    c.snapshot_budget_gb = float(getattr(p, "snapshot_budget_gb", 0.0))
    c.checkpoint_slots = int(getattr(p, "checkpoint_slots", 0))
    c.checkpoint_precision = int(getattr(p, "checkpoint_precision", 0))
    return c


class nl_we_op:
    """Non-linear wave-equation operator F: model -> data for one shot ``s``."""

    nmodels = 3

    def __init__(self, domain: Domain, allsrc: np.ndarray, s: int, par: Param, dt_data: float, device: int = 0):
        if domain.nmodels != self.nmodels:
            raise _lib.FwiError(_lib.FWI_ERR_ARG, f"{type(self).__name__} needs {self.nmodels} model parameters")
        self._domain = domain
        self._allsrc = np.ascontiguousarray(allsrc, dtype=np.float32)
        w = self._allsrc
        self._src = w if w.ndim == 1 else np.ascontiguousarray(w[s])
        self._par = par.copy()
        self._par.sxyz = [list(par.sxyz[s])]
        self._par.rxyz = [[list(r) for r in par.rxyz[s]]]
        self._par.ns = 1
        self.dt_data = float(dt_data)
        self.device = device
        lib = _lib.load()
        rx = np.ascontiguousarray(np.asarray(par.rxyz[s], dtype=np.float32).reshape(-1, 5))
        sx = np.ascontiguousarray(np.asarray(par.sxyz[s], dtype=np.float32)[:3])
        ncomp = 1 if self._src.ndim == 1 else self._src.shape[0]
        self._nr = rx.shape[0]
        self._nt_data = self._src.shape[-1]
        h = C.c_void_p()
        cp = to_cparam(self._par)
        _lib.check(lib.fwi_op_create(C.byref(h), device, C.byref(domain.grid()), self.nmodels, C.byref(cp),
                                     _lib.fptr(self._src), ncomp, self._nt_data, self.dt_data, _lib.fptr(sx),
                                     self._nr, _lib.fptr(rx)))
        self._h = h

    # -- shapes ----------------------------------------------------------
    @property
    def nrcomp(self) -> int:
        # DAS channels (gl > 0) record one strain component (analyzeGeometry, we_op.cpp:23)
        return 1 if self.nmodels == 2 or self._par.gl > 0 else 3

    @property
    def domain_shape(self):
        return self._domain.shape

    @property
    def range_shape(self):
        return (self.nrcomp, self._nr, self._nt_data)

    def info(self) -> _lib.OpInfo:
        inf = _lib.OpInfo()
        _lib.check(_lib.load().fwi_op_get_info(self._h, C.byref(inf)))
        return inf

    # -- raw forms (we_op.hpp:50-51) -------------------------------------
    def apply_forward(self, add: bool, pmod: np.ndarray, pdat: np.ndarray) -> None:
        _check_f32(pmod, self.domain_shape, "model")
        _check_f32(pdat, self.range_shape, "data")
        _lib.check(_lib.load().fwi_op_forward(self._h, int(add), _lib.fptr(pmod), _lib.fptr(pdat)))

    def apply_jacobianT(self, add: bool, pmod: np.ndarray, pmod0: np.ndarray, pdat: np.ndarray) -> None:
        nm = min(3, self.nmodels)
        _check_f32(pmod, (nm,) + self.domain_shape[1:], "gradient")
        _check_f32(pmod0, self.domain_shape, "model")
        _check_f32(pdat, self.range_shape, "data")
        _lib.check(_lib.load().fwi_op_jacobianT(self._h, int(add), _lib.fptr(pmod), _lib.fptr(pmod0),
                                                _lib.fptr(pdat)))

    # -- vector forms (we_op.hpp:41-49) ----------------------------------
    def forward(self, add: bool, mod: np.ndarray, dat: Optional[np.ndarray] = None) -> np.ndarray:
        mod = np.ascontiguousarray(mod, dtype=np.float32)
        if dat is None:
            dat = np.zeros(self.range_shape, dtype=np.float32)
        self.apply_forward(add, mod, dat)
        return dat

    def jacobianT(self, add: bool, mod: Optional[np.ndarray], mod0: np.ndarray, dat: np.ndarray) -> np.ndarray:
        nm = min(3, self.nmodels)
        if mod is None:
            mod = np.zeros((nm,) + self.domain_shape[1:], dtype=np.float32)
        self.apply_jacobianT(add, mod, np.ascontiguousarray(mod0, dtype=np.float32),
                             np.ascontiguousarray(dat, dtype=np.float32))
        return mod

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.load().fwi_op_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _check_f32(a: np.ndarray, shape, what: str) -> None:
    if not isinstance(a, np.ndarray) or a.dtype != np.float32 or not a.flags.c_contiguous:
        raise _lib.FwiError(_lib.FWI_ERR_ARG, f"{what} must be a C-contiguous float32 array")
    if tuple(a.shape) != tuple(shape) and a.size != int(np.prod(shape)):
        raise _lib.FwiError(_lib.FWI_ERR_ARG, f"{what} has shape {a.shape}, expected {tuple(shape)}")


class nl_we_op_e(nl_we_op):
    """Elastic isotropic operator (we_op.hpp:55-100); model (vp, vs, rho)."""

    nmodels = 3


class nl_we_op_vti(nl_we_op_e):
    """Elastic VTI operator (we_op.hpp:103-131); model (vp, vs, rho, delta, eps, gamma)."""

    nmodels = 6


class nl_we_op_a(nl_we_op_e):
    """Acoustic variable-density operator (we_op.hpp:134-167); model (vp, rho)."""

    nmodels = 2


def op_for(nmodels: int):
    return {2: nl_we_op_a, 3: nl_we_op_e, 6: nl_we_op_vti}[nmodels]


def from_survey(sv, s: int = 0, device: int = 0) -> nl_we_op:
    """Operator for shot ``s`` of a synth.Survey."""
    dom = Domain(sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.nmodels, sv.ox, sv.oy, sv.oz)
    return op_for(sv.nmodels)(dom, sv.wavelet, s, sv.par, sv.dt_data, device)


def forward_batch(sv, device: int = 0) -> np.ndarray:
    """Modeling of all shots of a survey on the shared model: [ns][nrcomp][nr][nt]."""
    lib = _lib.load()
    dom = Domain(sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.nmodels, sv.ox, sv.oy, sv.oz)
    ns = len(sv.par.sxyz)
    nr = len(sv.par.rxyz[0])
    if any(len(r) != nr for r in sv.par.rxyz):
        raise _lib.FwiError(_lib.FWI_ERR_ARG, "forward_batch needs the same receiver count for every shot")
    w = np.ascontiguousarray(sv.wavelet, dtype=np.float32)
    ncomp = 1 if w.ndim == 1 else w.shape[0]
    sx = np.ascontiguousarray(np.asarray(sv.par.sxyz, dtype=np.float32)[:, :3])
    rx = np.ascontiguousarray(np.asarray(sv.par.rxyz, dtype=np.float32).reshape(ns, nr, 5))
    nrcomp = 1 if sv.nmodels == 2 or sv.par.gl > 0 else 3  # DAS: strain along each fibre
    out = np.zeros((ns, nrcomp, nr, w.shape[-1]), dtype=np.float32)
    model = np.ascontiguousarray(sv.model, dtype=np.float32)
    cp = to_cparam(sv.par)
    _lib.check(lib.fwi_forward_batch(device, C.byref(dom.grid()), sv.nmodels, C.byref(cp), _lib.fptr(model),
                                     _lib.fptr(w), ncomp, w.shape[-1], sv.dt_data, ns, _lib.fptr(sx), nr,
                                     _lib.fptr(rx), _lib.fptr(out)))
    return out


class FwiObjective:
    """FWI objective of all shots of a survey on the device (the reference's
    nlls_fwi, optimization.cpp:5-197): ``evaluate(model)`` returns the misfit
    (FP64), the gradient in the model's parametrisation and the residuals.

    ``batch`` shots advance in lockstep per launch; ``sv.par.snapshot_storage``
    selects FP32 or FP16 second-difference snapshot storage."""

    def __init__(self, sv, observed: np.ndarray, normalize: bool = True, batch: Optional[int] = None,
                 device: int = 0):
        lib = _lib.load()
        self.sv = sv
        self.ns = len(sv.par.sxyz)
        self.nr = len(sv.par.rxyz[0])
        if any(len(r) != self.nr for r in sv.par.rxyz):
            raise _lib.FwiError(_lib.FWI_ERR_ARG, "every shot needs the same receiver count")
        self.nm = min(3, sv.nmodels)
        w = np.ascontiguousarray(sv.wavelet, dtype=np.float32)
        ncomp = 1 if w.ndim == 1 else w.shape[0]
        self.nt_data = w.shape[-1]
        self.nrcomp = 1 if sv.nmodels == 2 or sv.par.gl > 0 else 3  # DAS: strain along each fibre
        obs = np.ascontiguousarray(observed, dtype=np.float32)
        if obs.size != self.ns * self.nrcomp * self.nr * self.nt_data:
            raise _lib.FwiError(_lib.FWI_ERR_ARG, f"observed data of shape {obs.shape} do not match the survey")
        sx = np.ascontiguousarray(np.asarray(sv.par.sxyz, dtype=np.float32)[:, :3])
        rx = np.ascontiguousarray(np.asarray(sv.par.rxyz, dtype=np.float32).reshape(self.ns, self.nr, 5))
        dom = Domain(sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.nmodels, sv.ox, sv.oy, sv.oz)
        self.shape = dom.shape
        cp = to_cparam(sv.par)
        h = C.c_void_p()
        _lib.check(lib.fwi_objective_create(C.byref(h), device, C.byref(dom.grid()), sv.nmodels, C.byref(cp),
                                            _lib.fptr(w), ncomp, self.nt_data, sv.dt_data, self.ns, _lib.fptr(sx),
                                            self.nr, _lib.fptr(rx), _lib.fptr(obs), int(bool(normalize)),
                                            int(batch or self.ns)))
        self._h = h

    def evaluate(self, model: np.ndarray, want_residual: bool = False):
        m = np.ascontiguousarray(model, dtype=np.float32)
        if m.size != int(np.prod(self.shape)):
            raise _lib.FwiError(_lib.FWI_ERR_ARG, f"model of shape {m.shape}, expected {self.shape}")
        g = np.zeros((self.nm,) + tuple(self.shape[1:]), dtype=np.float32)
        r = np.zeros((self.ns, self.nrcomp, self.nr, self.nt_data), dtype=np.float32) if want_residual else None
        f = C.c_double()
        _lib.check(_lib.load().fwi_objective_evaluate(self._h, _lib.fptr(m), C.byref(f), _lib.fptr(g),
                                                      _lib.fptr(r) if r is not None else None))
        return (f.value, g, r) if want_residual else (f.value, g)

    def evaluate_shots(self, model: np.ndarray):
        """One objective per shot from the same batched launches: misfits
        [ns] (FP64) and gradients [ns][nm][...], each shot normalised by its
        own data (independent gradient requests on one model)."""
        m = np.ascontiguousarray(model, dtype=np.float32)
        if m.size != int(np.prod(self.shape)):
            raise _lib.FwiError(_lib.FWI_ERR_ARG, f"model of shape {m.shape}, expected {self.shape}")
        g = np.zeros((self.ns, self.nm) + tuple(self.shape[1:]), dtype=np.float32)
        f = np.zeros(self.ns, dtype=np.float64)
        _lib.check(_lib.load().fwi_objective_evaluate_shots(self._h, _lib.fptr(m),
                                                            f.ctypes.data_as(C.POINTER(C.c_double)), _lib.fptr(g)))
        return f, g

    def set_shots(self, sv, observed: np.ndarray) -> None:
        """New shots (same counts) for the next evaluations, which reuse the
        objective's device buffers."""
        if len(sv.par.sxyz) != self.ns or any(len(r) != self.nr for r in sv.par.rxyz):
            raise _lib.FwiError(_lib.FWI_ERR_ARG, "set_shots keeps the shot and receiver counts")
        obs = np.ascontiguousarray(observed, dtype=np.float32)
        if obs.size != self.ns * self.nrcomp * self.nr * self.nt_data:
            raise _lib.FwiError(_lib.FWI_ERR_ARG, f"observed data of shape {obs.shape} do not match the survey")
        sx = np.ascontiguousarray(np.asarray(sv.par.sxyz, dtype=np.float32)[:, :3])
        rx = np.ascontiguousarray(np.asarray(sv.par.rxyz, dtype=np.float32).reshape(self.ns, self.nr, 5))
        _lib.check(_lib.load().fwi_objective_set_shots(self._h, _lib.fptr(sx), _lib.fptr(rx), _lib.fptr(obs)))
        self.sv = sv

    def device_bytes(self) -> int:
        return int(_lib.load().fwi_objective_device_bytes(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.load().fwi_objective_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
