"""Seeded synthetic surveys with the shapes of the benchmark configurations.

There are no public datasets for this path: every model, wavelet and
acquisition geometry is generated here from a seeded ``numpy`` generator, so
the GPU path and the CPU oracle read identical bytes.

Conventions (all as in the reference): units km, km/s, g/cc, s; model layout
``[nmodels][ny][nx][nz]`` with z fastest (``we_op.cpp:28-30``); acoustic models
hold (vp, rho), elastic (vp, vs, rho), VTI (vp, vs, rho, delta, epsilon,
gamma) -- the order ``analyzeModel`` expects (``we_op.cpp:247-251``).

Gaussian random fields are white noise smoothed by a Gaussian of the stated
correlation length (in cells) and rescaled to the stated standard deviation.
The Ricker wavelet is ``(1-2a)exp(-a)``, ``a=(pi f0 (t-t0))^2``, ``t0=1.2/f0``,
sampled at the propagation step.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .param import Param


def ricker(f0: float, dt: float, nt: int, t0: Optional[float] = None) -> np.ndarray:
    t0 = 1.2 / f0 if t0 is None else t0
    t = np.arange(nt, dtype=np.float64) * dt
    a = (np.pi * f0 * (t - t0)) ** 2
    return ((1.0 - 2.0 * a) * np.exp(-a)).astype(np.float32)


def grf(rng: np.random.Generator, shape, corr_cells: float, sigma: float) -> np.ndarray:
    """Zero-mean Gaussian random field with std ``sigma`` (float64)."""
    from scipy.ndimage import gaussian_filter

    w = rng.standard_normal(shape)
    if corr_cells > 0:
        w = gaussian_filter(w, sigma=corr_cells, mode="reflect")
    s = w.std()
    return w * (sigma / s if s > 0 else 0.0)


def gardner(vp_kms: np.ndarray) -> np.ndarray:
    """rho [g/cc] = 0.31 * vp[m/s]^0.25."""
    return 0.31 * np.power(1000.0 * vp_kms, 0.25)


@dataclass
class Survey:
    """One synthetic problem: model, wavelet, shots and receivers."""

    name: str
    nmodels: int
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    model: np.ndarray                 # float32 [nmodels][ny][nx][nz]
    wavelet: np.ndarray               # float32 [nt] (duplicated per analyzeWavelet) or [ncomp][nt]
    dt_data: float
    par: Param
    ox: float = 0.0
    oy: float = 0.0
    oz: float = 0.0
    extra: dict = field(default_factory=dict)

    @property
    def nt_data(self) -> int:
        return int(self.wavelet.shape[-1])

    @property
    def nxyz(self) -> int:
        return self.nx * self.ny * self.nz

    def shot(self, s: int) -> "Survey":
        """A one-shot view (shot s), the unit the operator works on."""
        p = self.par.copy()
        p.sxyz = [list(self.par.sxyz[s])]
        p.rxyz = [[list(r) for r in self.par.rxyz[s]]]
        p.ns = 1
        return Survey(self.name + f"/shot{s}", self.nmodels, self.nx, self.ny, self.nz, self.dx, self.dy,
                      self.dz, self.model, self.wavelet, self.dt_data, p, self.ox, self.oy, self.oz,
                      dict(self.extra))


def _grid_receivers(ixs, iys, z, dx, dy) -> List[List[float]]:
    return [[float(ix * dx), float(iy * dy), float(z), 0.0, 0.0] for iy in iys for ix in ixs]


def acoustic_linear(n: int = 101, nsteps: int = 1000, d: float = 0.01, dt: float = 0.001,
                    f0: float = 15.0, seed: int = 1, taper: int = 20, rec_stride: int = 2,
                    rec_iz: int = 2) -> Survey:
    """Acoustic variable-density modeling: vp linear in depth 1.5->3.0 km/s plus
    a seeded GRF (sigma 0.05 km/s, 5-cell correlation), Gardner density,
    free-surface top, absorbing elsewhere with ``taper``-point tapers, one 15 Hz
    Ricker pressure source at grid (n/2, n/2, 5), surface receivers every
    ``rec_stride`` points at depth index ``rec_iz``."""
    rng = np.random.default_rng(seed)
    nx = ny = nz = n
    iz = np.arange(nz, dtype=np.float64)
    vp = 1.5 + 1.5 * iz / (nz - 1)
    vp = np.broadcast_to(vp, (ny, nx, nz)) + grf(rng, (ny, nx, nz), 5.0, 0.05)
    rho = gardner(vp)
    model = np.stack([vp, rho]).astype(np.float32)
    par = Param(nmodels=2, resampling="sinc", courant=0.5, dt=-1.0, sub=0)
    par.set_bc(1, 2, 2, 2, 2, 2).set_taper(0, taper, taper, taper, taper, taper)
    c = n // 2
    par.sxyz = [[c * d, c * d, 5 * d]]
    idx = list(range(0, n, rec_stride))
    par.rxyz = [_grid_receivers(idx, idx, rec_iz * d, d, d)]
    par.ns = 1
    w = ricker(f0, dt, nsteps + 1)
    return Survey(f"acoustic_linear_{n}", 2, nx, ny, nz, d, d, d, model, w, dt, par)


def layered_background(nx, ny, nz, vtop, vbot, nlayers, vs_ratio, rng, pert=0.03, corr=8.0):
    """Flat layers with vp from vtop to vbot, vs = vp/vs_ratio, Gardner rho, all
    multiplied by (1 + GRF) of std ``pert``/2 (so ~95% within +-pert)."""
    bounds = np.linspace(0, nz, nlayers + 1).astype(int)
    vlay = np.linspace(vtop, vbot, nlayers)
    vp1 = np.empty(nz)
    for k in range(nlayers):
        vp1[bounds[k]:bounds[k + 1]] = vlay[k]
    vp = np.broadcast_to(vp1, (ny, nx, nz)).copy()
    if pert > 0:
        vp *= 1.0 + grf(rng, (ny, nx, nz), corr, pert / 2.0)
    vs = vp / vs_ratio
    rho = gardner(vp)
    return vp, vs, rho


def elastic_layered(n: int = 256, nsteps: int = 3000, d: float = 0.008, dt: float = 0.0006,
                    f0: float = 12.0, seed: int = 2, nshots: int = 8, taper: int = 20,
                    rec_stride: int = 2) -> Survey:
    """Elastic isotropic modeling: 6 flat layers vp 1.8->4.5 km/s, vs=vp/1.8,
    Gardner rho, x(1+GRF +-3%); explosive moment-tensor sources (mxx=myy=mzz=1)
    on a 2x4 grid at 16 m depth; 3-component particle-velocity receivers every
    ``rec_stride`` points on the surface."""
    rng = np.random.default_rng(seed)
    nx = ny = nz = n
    vp, vs, rho = layered_background(nx, ny, nz, 1.8, 4.5, 6, 1.8, rng)
    model = np.stack([vp, vs, rho]).astype(np.float32)
    par = Param(nmodels=3, mt=True, mxx=1, myy=1, mzz=1, mxy=0, mxz=0, myz=0, seismotype=1, sub=0)
    par.set_bc(1, 2, 2, 2, 2, 2).set_taper(0, taper, taper, taper, taper, taper)
    xs = [n // 4, 3 * n // 4]
    ys = [n // 8, 3 * n // 8, 5 * n // 8, 7 * n // 8]
    shots = [[x * d, y * d, 0.016] for y in ys for x in xs][:nshots]
    idx = list(range(0, n, rec_stride))
    rec = _grid_receivers(idx, idx, 0.0, d, d)
    par.sxyz = shots
    par.rxyz = [rec for _ in shots]
    par.ns = len(shots)
    w = ricker(f0, dt, nsteps + 1)
    return Survey(f"elastic_layered_{n}", 3, nx, ny, nz, d, d, d, model, w, dt, par)


def elastic_anomaly(n: int = 200, nsteps: int = 2500, d: float = 0.01, dt: float = 0.001,
                    f0: float = 10.0, seed: int = 3, nshots_side: int = 4, taper: int = 20,
                    rec_stride: int = 2, smooth_km: float = 0.2) -> Survey:
    """Elastic FWI problem: layered background + three Gaussian vp/vs anomalies
    (+-8%, radius 0.15 km) as the true model; the initial model is the true one
    smoothed with a Gaussian of ``smooth_km``.  ``model`` holds the initial
    model, ``extra['true_model']`` the true one."""
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    nx = ny = nz = n
    vp, vs, rho = layered_background(nx, ny, nz, 1.8, 4.5, 6, 1.8, rng, pert=0.0)
    L = (n - 1) * d
    y, x, z = np.meshgrid(np.arange(ny) * d, np.arange(nx) * d, np.arange(nz) * d, indexing="ij")
    centres = [(0.3 * L, 0.4 * L, 0.5 * L, +0.08), (0.7 * L, 0.6 * L, 0.45 * L, -0.08),
               (0.5 * L, 0.5 * L, 0.7 * L, +0.08)]
    r0 = 0.15
    for cx, cy, cz, a in centres:
        g = np.exp(-((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) / (2 * r0 ** 2))
        vp = vp * (1 + a * g)
        vs = vs * (1 + a * g)
    true = np.stack([vp, vs, rho]).astype(np.float32)
    sig = smooth_km / d
    init = np.stack([gaussian_filter(true[i].astype(np.float64), sig, mode="nearest")
                     for i in range(3)]).astype(np.float32)
    par = Param(nmodels=3, mt=False, fangle=np.pi / 2, fazimuth=0.0, seismotype=0, sub=-1)
    par.set_bc(1, 2, 2, 2, 2, 2).set_taper(0, taper, taper, taper, taper, taper)
    pos = [(k + 0.5) * n / nshots_side for k in range(nshots_side)]
    shots = [[px * d, py * d, 0.02] for py in pos for px in pos]
    idx = list(range(0, n, rec_stride))
    rec = _grid_receivers(idx, idx, 0.0, d, d)
    par.sxyz = shots
    par.rxyz = [rec for _ in shots]
    par.ns = len(shots)
    w = ricker(f0, dt, nsteps + 1)
    return Survey(f"elastic_anomaly_{n}", 3, nx, ny, nz, d, d, d, init, w, dt, par,
                  extra={"true_model": true})


def vti_layered(nx: int = 320, ny: int = 320, nz: int = 200, nsteps: int = 3000, d: float = 0.01,
                dt: float = 0.0008, f0: float = 10.0, seed: int = 4, nshots: int = 24, taper: int = 20,
                rec_stride: int = 2) -> Survey:
    """Elastic VTI: layered vp 2.0->4.2 km/s, vs=vp/1.9, Gardner rho, Thomsen
    epsilon 0->0.20 and delta 0->0.10 layered plus smooth GRF, gamma=0; vertical
    force sources on a 4x6 grid; 3-component displacement receivers."""
    rng = np.random.default_rng(seed)
    vp, vs, rho = layered_background(nx, ny, nz, 2.0, 4.2, 6, 1.9, rng, pert=0.0)
    bounds = np.linspace(0, nz, 7).astype(int)
    eps1 = np.empty(nz)
    del1 = np.empty(nz)
    for k, (e, dl) in enumerate(zip(np.linspace(0, 0.2, 6), np.linspace(0, 0.1, 6))):
        eps1[bounds[k]:bounds[k + 1]] = e
        del1[bounds[k]:bounds[k + 1]] = dl
    eps = np.clip(np.broadcast_to(eps1, (ny, nx, nz)) + grf(rng, (ny, nx, nz), 10.0, 0.01), 0, None)
    dlt = np.broadcast_to(del1, (ny, nx, nz)) + grf(rng, (ny, nx, nz), 10.0, 0.005)
    gam = np.zeros((ny, nx, nz))
    model = np.stack([vp, vs, rho, dlt, eps, gam]).astype(np.float32)
    par = Param(nmodels=6, mt=False, fangle=np.pi / 2, seismotype=0, sub=0)
    par.set_bc(1, 2, 2, 2, 2, 2).set_taper(0, taper, taper, taper, taper, taper)
    xs = [(k + 0.5) * nx / 4 for k in range(4)]
    ys = [(k + 0.5) * ny / 6 for k in range(6)]
    shots = [[x * d, y * d, 0.02] for y in ys for x in xs][:nshots]
    rec = _grid_receivers(list(range(0, nx, rec_stride)), list(range(0, ny, rec_stride)), 0.0, d, d)
    par.sxyz = shots
    par.rxyz = [rec for _ in shots]
    par.ns = len(shots)
    w = ricker(f0, dt, nsteps + 1)
    return Survey(f"vti_layered_{nx}x{ny}x{nz}", 6, nx, ny, nz, d, d, d, model, w, dt, par)
