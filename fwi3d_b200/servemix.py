"""Seeded request mixes for the serving loop (the serving configuration of
the benchmark, scaled): Poisson arrivals, models of the three physics at
uneven grid sizes, modeling and gradient shots."""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

from . import ops, serving, synth


def _model(kind: str, n: Tuple[int, int, int], seed: int):
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    d = 0.01
    if kind == "acoustic":
        iz = np.arange(nz, dtype=np.float64)
        vp = np.broadcast_to(1.5 + 1.5 * iz / (nz - 1), (ny, nx, nz)) + synth.grf(rng, (ny, nx, nz), 5.0, 0.05)
        return np.stack([vp, synth.gardner(vp)]).astype(np.float32), 2
    vp, vs, rho = synth.layered_background(nx, ny, nz, 1.8, 4.5, 6, 1.8, rng)
    if kind == "elastic":
        return np.stack([vp, vs, rho]).astype(np.float32), 3
    eps = np.clip(0.1 + synth.grf(rng, (ny, nx, nz), 10.0, 0.02), 0, None)
    dlt = 0.05 + synth.grf(rng, (ny, nx, nz), 10.0, 0.01)
    return np.stack([vp, vs, rho, dlt, eps, np.zeros_like(vp)]).astype(np.float32), 6


# The bench's serving mix: grids from the lower part of the configuration's
# range (96^3 .. 384x384x256), time axes of 1000-2000 steps (of 1000-4000),
# receiver lines of 48-96 (of 64-192) per side, so that a mix of a few dozen
# requests runs in about a minute.
BENCH_GRIDS = ((96, 96, 96), (160, 144, 128), (224, 192, 160))
BENCH_STEPS = (1000, 1500, 2000)
BENCH_REC = (48, 64, 96)
# checkpoint slots of a gradient request (FP32 restart states, binomial schedule)
GRADIENT_SLOTS = 40


def make_mix(nreq: int = 48, rate: float = 20.0, seed: int = 5, grids=((64, 64, 64), (96, 96, 80), (128, 112, 96)),
             steps=(200, 300, 400), rec=(16, 24), p_gradient: float = 0.25):
    """Returns (models, requests).  Six models (acoustic, elastic, VTI, two
    grids each), each request one shot on a random model with a 8-15 Hz
    Ricker, steps and receiver lines drawn from small sets (so that shots of
    the same model can share a batch), mode gradient with `p_gradient`
    (FP32 checkpoints with GRADIENT_SLOTS slots when the time axis is longer
    than 500 steps)."""
    rng = np.random.default_rng(seed)
    kinds = ["acoustic", "elastic", "vti"]
    models: Dict[str, np.ndarray] = {}
    meta = {}
    for k, kind in enumerate(kinds):
        for j in range(2):
            g = grids[(k + j) % len(grids)]
            m, nm = _model(kind, g, seed * 10 + 2 * k + j)
            mid = f"{kind}{j}"
            models[mid] = m
            meta[mid] = (g, nm)
    t = 0.0
    reqs: List[serving.Request] = []
    for i in range(nreq):
        t += rng.exponential(1.0 / rate)
        mid = list(models)[rng.integers(len(models))]
        (nx, ny, nz), nm = meta[mid]
        nsteps = int(rng.choice(steps))
        f0 = float(rng.uniform(8.0, 15.0))
        nrl = int(rng.choice(rec))
        mode = "gradient" if rng.random() < p_gradient else "modeling"
        d, dt = 0.01, 0.001
        par = synth.Param(nmodels=nm, sub=-1, seismotype=0, mt=False, fangle=np.pi / 2)
        par.set_bc(1, 2, 2, 2, 2, 2).set_taper(0, 10, 10, 10, 10, 10)
        sx = [float(rng.uniform(0.2, 0.8)) * (nx - 1) * d, float(rng.uniform(0.2, 0.8)) * (ny - 1) * d, 0.02]
        ix = np.linspace(0, nx - 1, nrl).astype(int)
        iy = np.linspace(0, ny - 1, nrl).astype(int)
        par.sxyz = [sx]
        par.rxyz = [[[float(a * d), float(b * d), 0.0, 0.0, 0.0] for b in iy for a in ix]]
        par.ns = 1
        w = synth.ricker(round(f0), dt, nsteps + 1)  # f0 rounded so that same-model shots may batch
        sv = synth.Survey(f"{mid}_{i}", nm, nx, ny, nz, d, d, d, models[mid], w, dt, par)
        if mode == "gradient" and nsteps > 500:
            sv.par.checkpoint_slots = GRADIENT_SLOTS
        r = serving.Request(i, mid, mode, sv, arrival=t)
        reqs.append(r)
    # observed data of the gradient requests: the model with a 3 % slower top half
    for r in reqs:
        if r.mode == "gradient":
            sv = r.survey
            true = models[r.model_id].copy()
            true[0, :, :, : sv.nz // 2] *= 0.97
            tv = synth.Survey(sv.name, sv.nmodels, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, true, sv.wavelet,
                              sv.dt_data, sv.par.copy())
            r.observed = ops.forward_batch(tv)
    return models, reqs
