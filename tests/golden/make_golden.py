"""Generate the golden fixtures of tests/golden/ from the reference itself.

The reference (nmbader/fwi3d) ships no tests or golden vectors, so these are
outputs of its own CPU library -- built from its sources by oracle/Makefile
into oracle/_ref -- on seeded synthetic inputs (fwi3d_b200.synth).  Each
fixture stores the generator arguments, the FP32-build output and the
FP64-build output (the error oracle).  Regenerate with

    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fwi3d_b200 import synth  # noqa: E402
from oracle import refpy  # noqa: E402

# name -> (builder, kwargs, overrides applied to par, gradient?)
CASES = {
    "acoustic_24": ("acoustic_linear", dict(n=24, nsteps=120, taper=6, rec_stride=3),
                    dict(bc=(1, 2, 2, 2, 2, 2)), False),
    "acoustic_rigid_24": ("acoustic_linear", dict(n=24, nsteps=120, taper=4, rec_stride=4),
                          dict(bc=(3, 1, 2, 3, 2, 1)), False),
    "elastic_mt_24": ("elastic_layered", dict(n=24, nsteps=100, taper=6, rec_stride=3, nshots=1),
                      dict(bc=(1, 2, 2, 2, 2, 2), sxyz=(0.5, 0.4, 0.3)), False),
    "elastic_force_24": ("elastic_layered", dict(n=24, nsteps=100, taper=5, rec_stride=4, nshots=1),
                         dict(bc=(2, 1, 2, 1, 2, 1), mt=False, sxyz=(0.45, 0.5, 0.35)), False),
    "vti_24": ("vti_layered", dict(nx=24, ny=26, nz=22, nsteps=100, taper=5, rec_stride=3, nshots=1, dt=0.0005),
               dict(bc=(1, 2, 2, 2, 2, 2), sxyz=(0.5, 0.4, 0.3)), False),
    "grad_acoustic_20": ("acoustic_linear", dict(n=20, nsteps=80, taper=4, rec_stride=3),
                         dict(bc=(1, 2, 2, 2, 2, 2), sub=1), True),
    "grad_elastic_20": ("elastic_layered", dict(n=20, nsteps=70, taper=4, rec_stride=3, nshots=1),
                        dict(bc=(1, 2, 2, 2, 2, 2), sxyz=(0.5, 0.4, 0.3), sub=1), True),
    "grad_vti_20": ("vti_layered", dict(nx=20, ny=22, nz=20, nsteps=71, taper=4, rec_stride=3, nshots=1, dt=0.0005),
                    dict(bc=(2, 1, 2, 1, 2, 1), sxyz=(0.5, 0.4, 0.3), sub=2), True),
}


def build(name):
    builder, kw, ov, grad = CASES[name]
    sv = getattr(synth, builder)(**kw)
    p = sv.par
    if "bc" in ov:
        p.set_bc(*ov["bc"])
    if "mt" in ov:
        p.mt = ov["mt"]
    if "sub" in ov:
        p.sub = ov["sub"]
    if "sxyz" in ov:
        fx, fy, fz = ov["sxyz"]
        p.sxyz = [[fx * (sv.nx - 1) * sv.dx, fy * (sv.ny - 1) * sv.dy, fz * (sv.nz - 1) * sv.dz]]
    return sv, grad


def adjoint_data(shape, scale, seed=7):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(shape) * scale).astype(np.float32)


def main():
    index = {}
    for name in CASES:
        sv, grad = build(name)
        d32, info = refpy.modeling(sv, precision="fp32")
        d64, _ = refpy.modeling(sv, precision="fp64")
        out = {"traces_fp32": d32.astype(np.float32), "traces_fp64": d64}
        if grad:
            adj = adjoint_data(d32.shape, float(np.abs(d32).max()))
            _, g32, _ = refpy.forward_jacobianT(sv, adj, precision="fp32")
            _, g64, _ = refpy.forward_jacobianT(sv, adj, precision="fp64")
            out["grad_fp32"] = g32.astype(np.float32)
            out["grad_fp64"] = g64
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        index[name] = {"dt": info.dt, "nt": info.nt, "sub": info.sub}
        print(name, {k: v.shape for k, v in out.items()}, index[name])
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
