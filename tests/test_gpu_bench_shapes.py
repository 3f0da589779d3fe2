"""GPU parity on grids that run the benchmark's kernels.

The elastic step splits each time step into tiles that hold no SBP closure row
along x or z (interior tiles), tiles next to an x or z face (edge tiles), the
six planes next to each y wall, and the SAT of the faces.  The grids here are
large enough in x and z for interior tiles (an axis holds one when it is at
least one tile plus two closure widths long), use several y chunks, and place
sources in the interior so that the wave crosses interior tiles, edge tiles and
the wall slabs within the window.  Receivers fill a 3-D lattice so that the
traces sample the volume, not only the surface.

Tolerances (as in the other parity tests): traces within 1e-5 relative L2 of
the reference's FP32 build, gradients within 1e-4; the FP64 build's distance is
printed beside each.  The benchmark configurations (elastic 256^3, VTI
320x320x200) are checked on short windows of their full grids.
"""
import numpy as np
import pytest

from fwi3d_b200 import ops, synth

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5
GRAD_TOL = 1e-4


def rel(a, b):
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _lattice(nx, ny, nz, d, stride, lo=1):
    """Receivers every ``stride`` points on each axis, from ``lo`` to the far face."""
    xs = list(range(lo, nx, stride)) + [nx - 2]
    ys = list(range(lo, ny, stride)) + [ny - 2]
    zs = list(range(lo, nz, stride)) + [nz - 2]
    return [[float(ix * d), float(iy * d), float(iz * d), 0.0, 0.0] for iy in ys for ix in xs for iz in zs]


def _crop(sv, nx, ny, nz):
    sv.model = np.ascontiguousarray(sv.model[:, :ny, :nx, :nz])
    sv.nx, sv.ny, sv.nz = nx, ny, nz
    return sv


def _early_ricker(sv, f0, nsteps, dt):
    """A Ricker wavelet centred early (t0 = 0.8/f0) so that short windows carry energy."""
    sv.wavelet = synth.ricker(f0, dt, nsteps + 1, t0=0.8 / f0)
    sv.dt_data = dt
    return sv


def elastic_box(nx, ny, nz, steps, nshots=1, mt=True, stride=7):
    n = max(nx, ny, nz)
    sv = synth.elastic_layered(n=n, nsteps=steps, d=0.008, dt=0.0006, taper=8, rec_stride=4, nshots=1)
    _crop(sv, nx, ny, nz)
    sv.par.mt = mt
    if not mt:
        sv.par.fangle, sv.par.fazimuth = 0.6, 0.4
    d = sv.dx
    rng = np.random.default_rng(11)
    shots = []
    for s in range(nshots):
        fx, fy, fz = rng.uniform(0.3, 0.7, 3)
        shots.append([fx * (nx - 1) * d, fy * (ny - 1) * d, fz * (nz - 1) * d])
    rec = _lattice(nx, ny, nz, d, stride)
    sv.par.sxyz = shots
    sv.par.rxyz = [rec for _ in shots]
    sv.par.ns = nshots
    sv.par.seismotype = 0
    return _early_ricker(sv, 25.0, steps, 0.0006)


def vti_box(nx, ny, nz, steps, stride=7):
    sv = synth.vti_layered(nx=nx, ny=ny, nz=nz, nsteps=steps, d=0.01, dt=0.0008, taper=8, rec_stride=4,
                           nshots=1)
    d = sv.dx
    sv.par.sxyz = [[0.45 * (nx - 1) * d, 0.55 * (ny - 1) * d, 0.5 * (nz - 1) * d]]
    sv.par.rxyz = [_lattice(nx, ny, nz, d, stride)]
    sv.par.ns = 1
    return _early_ricker(sv, 20.0, steps, 0.0008)


def _check_modeling(oracle, sv, fp64=True):
    d = ops.forward_batch(sv) if sv.par.ns > 1 else ops.from_survey(sv).forward(False, sv.model)[None]
    for s in range(sv.par.ns):
        ref, _ = oracle.modeling(sv, shot=s, precision="fp32")
        e32 = rel(d[s], ref)
        msg = f"{sv.name} shot {s}: vs fp32 {e32:.3e}"
        if fp64:
            ref64, _ = oracle.modeling(sv, shot=s, precision="fp64")
            msg += f"  vs fp64 {rel(d[s], ref64):.3e}  fp32-vs-fp64 {rel(ref, ref64):.3e}"
        print(msg)
        assert np.abs(ref).max() > 0
        assert e32 < TRACE_TOL, msg


# (nx, ny, nz): interior tiles on x and z, several y chunks; nz = 101 is not a
# multiple of 4, so its planes are copied by per-thread asynchronous copies
# instead of tensor-map bulk copies
SHAPES = [(100, 76, 96), (63, 45, 101)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("mt", [True, False])
def test_elastic_interior_tiles(oracle_fp32, monkeypatch, shape, mt):
    monkeypatch.setenv("FWI_FUSED_WAVES", "64")  # as many y chunks as the planes allow
    sv = elastic_box(*shape, steps=170, mt=mt)
    _check_modeling(oracle_fp32, sv, fp64=mt)


def test_elastic_interior_tiles_batch(oracle_fp32, monkeypatch):
    """Three shots in one launch, each against its own oracle run."""
    monkeypatch.setenv("FWI_FUSED_WAVES", "64")
    sv = elastic_box(100, 76, 96, steps=150, nshots=3)
    _check_modeling(oracle_fp32, sv, fp64=False)


@pytest.mark.parametrize("shape", SHAPES)
def test_vti_interior_tiles(oracle_fp32, monkeypatch, shape):
    monkeypatch.setenv("FWI_FUSED_WAVES", "64")
    sv = vti_box(*shape, steps=150)
    _check_modeling(oracle_fp32, sv)


def _grad_check(oracle, sv, sub):
    sv.par.sub = sub
    rng = np.random.default_rng(5)
    ref, _ = oracle.modeling(sv, precision="fp32")
    adj = (rng.standard_normal(ref.shape) * np.abs(ref).max()).astype(np.float32)
    op = ops.from_survey(sv)
    syn = op.forward(False, sv.model)
    g = op.jacobianT(False, None, sv.model, adj)
    s32, g32, _ = oracle.forward_jacobianT(sv, adj, precision="fp32")
    _, g64, _ = oracle.forward_jacobianT(sv, adj, precision="fp64")
    assert rel(syn, s32) < TRACE_TOL
    for k in range(g32.shape[0]):
        e32, e64 = rel(g[k], g32[k]), rel(g[k], g64[k])
        print(f"{sv.name} grad[{k}]: vs fp32 {e32:.3e}  vs fp64 {e64:.3e}  fp32-vs-fp64 {rel(g32[k], g64[k]):.3e}")
        assert e32 < GRAD_TOL, f"parameter {k}"


def test_elastic_gradient_interior_tiles(oracle_fp32, monkeypatch):
    monkeypatch.setenv("FWI_FUSED_WAVES", "64")
    sv = elastic_box(72, 52, 80, steps=130, stride=9)
    _grad_check(oracle_fp32, sv, 1)


def test_vti_gradient_interior_tiles(oracle_fp32, monkeypatch):
    monkeypatch.setenv("FWI_FUSED_WAVES", "64")
    sv = vti_box(72, 52, 80, steps=120, stride=9)
    _grad_check(oracle_fp32, sv, 2)


# --- windows of the benchmark configurations, on their full grids ---

def test_config2_window(oracle_fp32):
    """Elastic isotropic 256^3 (8 m, dt 0.6 ms): 100 steps, one interior shot."""
    sv = elastic_box(256, 256, 256, steps=100, stride=16)
    sv.par.sxyz = [[128 * sv.dx, 120 * sv.dx, 124 * sv.dx]]
    _check_modeling(oracle_fp32, sv, fp64=False)


def test_config2_batch_matches_single_shots():
    """The benchmark's 8-shot batch on 256^3 gives the traces of eight one-shot
    operators (bitwise-identical kernels up to the batch index)."""
    sv = synth.elastic_layered(n=256, nsteps=200)
    _early_ricker(sv, 12.0, 200, 0.0006)
    batch = ops.forward_batch(sv)
    for s in range(sv.par.ns):
        single = ops.from_survey(sv, s).forward(False, sv.model)
        assert np.abs(single).max() > 0
        assert rel(batch[s], single) < 1e-6, f"shot {s}"


def test_config4_window(oracle_fp32):
    """VTI 320x320x200 (10 m, dt 0.8 ms): 40 steps, one interior shot."""
    sv = vti_box(320, 320, 200, steps=40, stride=16)
    sv.par.sxyz = [[160 * sv.dx, 150 * sv.dx, 100 * sv.dx]]
    _check_modeling(oracle_fp32, sv, fp64=False)
