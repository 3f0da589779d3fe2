"""Propagation parameters, mirroring the reference's ``struct param``.

Field names, meanings and defaults follow ``src/include/param.hpp:8-71`` of
nmbader/fwi3d for every knob the wave-propagation path reads.  Inversion-only
knobs (solver, regularisation, B-splines, file names) are not carried: they
belong to callers of the propagator, not to the propagator itself.

Units are the reference's: km, km/s, g/cc, s; moduli in GPa.
"""
from __future__ import annotations

import copy
import dataclasses
from dataclasses import dataclass, field
from typing import List

BC_NONE, BC_FREE_SURFACE, BC_ABSORBING, BC_RIGID = 0, 1, 2, 3


@dataclass
class Param:
    # time parameters (param.hpp:10-14)
    nt: int = 0
    sub: int = 0
    courant: float = 0.5
    dt: float = -1.0
    tmax: float = 0.0
    fmax: float = 10.0
    resampling: str = "sinc"
    sinc_half_length: int = 11

    # geometry (param.hpp:17-26); sxyz[s] = [x, y, z]; rxyz[s][r] = [x, y, z, dip, az]
    ns: int = 1
    nr: int = 1
    nscomp: int = 3
    nrcomp: int = 3
    sxyz: List[List[float]] = field(default_factory=list)
    rxyz: List[List[List[float]]] = field(default_factory=list)
    gl: float = 0.0

    # source mechanism and receiver type (param.hpp:33-37)
    mt: bool = False
    fangle: float = 0.0
    fazimuth: float = 0.0
    mxx: float = 1.0
    myy: float = 1.0
    mzz: float = 1.0
    mxy: float = 1.0
    mxz: float = 1.0
    myz: float = 1.0
    seismotype: int = 0

    # boundaries (param.hpp:40-41): 0 none, 1 free surface, 2 absorbing, 3 rigid
    bc_top: int = 1
    bc_bottom: int = 1
    bc_left: int = 1
    bc_right: int = 1
    bc_front: int = 1
    bc_back: int = 1
    taper_top: int = 0
    taper_bottom: int = 0
    taper_left: int = 0
    taper_right: int = 0
    taper_front: int = 0
    taper_back: int = 0
    free_surface_stiffness: float = 1.05
    taper_strength: float = 0.05

    # model bounds (param.hpp:44-45)
    vpmin: float = 0.2
    vpmax: float = 8.0
    vsmin: float = 0.1
    vsmax: float = 5.0
    rhomin: float = 0.1
    rhomax: float = 8.0
    deltamin: float = -0.5
    deltamax: float = 1.0
    epsilonmin: float = 0.0
    epsilonmax: float = 1.0
    gammamin: float = 0.0
    gammamax: float = 1.0
    vmax: float = 8.0
    vmin: float = 0.1

    nmodels: int = 3
    soft_clip: bool = False

    # miscellaneous (param.hpp:64-66)
    nthreads: int = 0
    verbose: int = 0

    # gradient snapshot storage (no reference counterpart): 0 FP32, 1 FP16
    # second-difference residuals with per-snapshot scales
    snapshot_storage: int = 0
    # HBM budget of that storage in GB (0: unlimited); above it, binomial
    # checkpointing with as many slots as fit
    snapshot_budget_gb: float = 0.0
    # binomial checkpointing (no reference counterpart): > 0 restart states
    # (prev, curr) kept on the device, whatever the budget; their storage
    # 0 FP32, 1 BF16, 2 FP16 (16-bit forms scaled per state, level, shot and
    # component by the field's max |value|)
    checkpoint_slots: int = 0
    checkpoint_precision: int = 0

    def copy(self) -> "Param":
        return copy.deepcopy(self)

    @property
    def bc(self) -> List[int]:
        return [self.bc_top, self.bc_bottom, self.bc_left, self.bc_right, self.bc_front, self.bc_back]

    @property
    def taper(self) -> List[int]:
        return [self.taper_top, self.taper_bottom, self.taper_left, self.taper_right,
                self.taper_front, self.taper_back]

    def set_bc(self, top, bottom, left, right, front, back) -> "Param":
        self.bc_top, self.bc_bottom, self.bc_left = top, bottom, left
        self.bc_right, self.bc_front, self.bc_back = right, front, back
        return self

    def set_taper(self, top, bottom, left, right, front, back) -> "Param":
        self.taper_top, self.taper_bottom, self.taper_left = top, bottom, left
        self.taper_right, self.taper_front, self.taper_back = right, front, back
        return self


def fields() -> List[str]:
    return [f.name for f in dataclasses.fields(Param)]
