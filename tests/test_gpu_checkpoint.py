"""Binomial checkpointing of the gradient's forward wavefield on the GPU.

The forward keeps `checkpoint_slots` restart states (prev, curr) of the batch;
the adjoint recomputes the states it needs from them in the order of the
Griewank-Walther schedule (revolve).  With FP32 checkpoints the recomputed
states are the forward's own, so the gradient equals the full-storage one;
with per-state scaled 16-bit checkpoints (BF16, FP16) the recomputation starts
from rounded states, and the gradient error against the reference's FP64 build
is measured and bounded here.
"""
import numpy as np
import pytest

from fwi3d_b200 import ops, synth

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _problem(n=28, steps=120, nside=2, sub=1):
    sv = synth.elastic_anomaly(n=n, nsteps=steps, nshots_side=nside, taper=6, rec_stride=3)
    sv.par.sub = sub
    true = synth.Survey(sv.name, sv.nmodels, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz,
                        sv.extra["true_model"], sv.wavelet, sv.dt_data, sv.par.copy())
    return sv, ops.forward_batch(true)


@pytest.mark.parametrize("slots", [2, 5, 17])
@pytest.mark.parametrize("steps,sub", [(120, 1), (121, 3)])
def test_fp32_checkpoints_equal_full_storage(slots, steps, sub):
    sv, obs = _problem(steps=steps, sub=sub)
    f0, g0 = ops.FwiObjective(sv, obs, batch=4).evaluate(sv.model)
    sv.par.checkpoint_slots = slots
    ck = ops.FwiObjective(sv, obs, batch=4)
    f1, g1 = ck.evaluate(sv.model)
    assert f1 == pytest.approx(f0, rel=1e-9)
    assert rel(g1, g0) < 1e-6
    # a second evaluation reuses the engine and its checkpoint slots
    f2, g2 = ck.evaluate(sv.model)
    assert f2 == pytest.approx(f0, rel=1e-9) and rel(g2, g0) < 1e-6


def test_budget_selects_checkpointing():
    """An HBM budget below full storage switches to checkpointing with as many
    slots as fit: same gradient, less device memory; a budget below the
    minimum is a clear error."""
    sv, obs = _problem()
    full = ops.FwiObjective(sv, obs, batch=4)
    f0, g0 = full.evaluate(sv.model)
    sv.par.snapshot_budget_gb = 0.03
    ck = ops.FwiObjective(sv, obs, batch=4)
    f1, g1 = ck.evaluate(sv.model)
    assert f1 == pytest.approx(f0, rel=1e-9) and rel(g1, g0) < 1e-6
    assert ck.device_bytes() < 0.5 * full.device_bytes()
    sv.par.snapshot_budget_gb = 0.001
    with pytest.raises(Exception, match="snapshot budget"):
        ops.FwiObjective(sv, obs, batch=4).evaluate(sv.model)


# 16-bit checkpoint error bounds (relative L2 per parameter, against the
# reference's FP64 build).  A restart from a rounded state adds grid-scale
# noise to the recomputed wavefield; its time and space derivatives, which the
# imaging condition takes, are not small against those of the wave, so the
# gradient error is far above the rounding unit (FP16 keeps 11 significant
# bits, BF16 8).  The FP32 path itself is a few 1e-6 from the FP64 build.
BOUND = {1: 5e-2, 2: 1e-2}


@pytest.mark.parametrize("precision", [1, 2])
def test_scaled_16bit_checkpoints_vs_fp64_oracle(oracle_fp32, precision):
    sv = synth.elastic_layered(n=28, nsteps=200, taper=6, rec_stride=3, nshots=1)
    sv.par.sxyz = [[0.5 * 28 * sv.dx, 0.4 * 28 * sv.dx, 0.3 * 28 * sv.dx]]
    sv.par.sub = 1
    rng = np.random.default_rng(0)
    ref, _ = oracle_fp32.modeling(sv, precision="fp32")
    adj = (rng.standard_normal(ref.shape) * np.abs(ref).max()).astype(np.float32)
    _, g64, _ = oracle_fp32.forward_jacobianT(sv, adj, precision="fp64")
    op = ops.from_survey(sv)
    op.forward(False, sv.model)
    g32 = op.jacobianT(False, None, sv.model, adj)
    sv.par.checkpoint_slots = 6
    sv.par.checkpoint_precision = precision
    op16 = ops.from_survey(sv)
    op16.forward(False, sv.model)
    g16 = op16.jacobianT(False, None, sv.model, adj)
    errs = []
    for k in range(3):
        e, e32 = rel(g16[k], g64[k]), rel(g32[k], g64[k])
        print(f"precision {precision} grad[{k}]: vs fp64 {e:.3e} (FP32 full storage {e32:.3e})")
        errs.append(e)
    assert max(errs) < BOUND[precision]


def _vti_case(n=26, steps=160):
    sv = synth.vti_layered(nx=n, ny=n + 2, nz=n - 2, nsteps=steps, taper=5, rec_stride=3, nshots=1, dt=0.0005)
    sv.par.sxyz = [[0.5 * n * sv.dx, 0.45 * n * sv.dx, 0.3 * n * sv.dx]]
    sv.par.sub = 1
    return sv


def test_vti_fp32_checkpoints_equal_full_storage():
    sv = _vti_case()
    rng = np.random.default_rng(1)
    op = ops.from_survey(sv)
    d = op.forward(False, sv.model)
    adj = (rng.standard_normal(d.shape) * np.abs(d).max()).astype(np.float32)
    g_full = op.jacobianT(False, None, sv.model, adj)
    sv.par.checkpoint_slots = 7
    opc = ops.from_survey(sv)
    opc.forward(False, sv.model)
    g_ck = opc.jacobianT(False, None, sv.model, adj)
    for k in range(3):
        assert rel(g_ck[k], g_full[k]) < 1e-6, k


@pytest.mark.parametrize("precision", [1, 2])
def test_vti_scaled_16bit_checkpoints_vs_fp64_oracle(oracle_fp32, precision):
    """The VTI gradient with 16-bit restart states (the configuration's FP16
    per-snapshot-scaled checkpoints) against the reference's FP64 build; the
    distance is printed and bounded as for the isotropic case."""
    sv = _vti_case()
    rng = np.random.default_rng(0)
    ref, _ = oracle_fp32.modeling(sv, precision="fp32")
    adj = (rng.standard_normal(ref.shape) * np.abs(ref).max()).astype(np.float32)
    _, g64, _ = oracle_fp32.forward_jacobianT(sv, adj, precision="fp64")
    op = ops.from_survey(sv)
    op.forward(False, sv.model)
    g32 = op.jacobianT(False, None, sv.model, adj)
    sv.par.checkpoint_slots = 6
    sv.par.checkpoint_precision = precision
    op16 = ops.from_survey(sv)
    op16.forward(False, sv.model)
    g16 = op16.jacobianT(False, None, sv.model, adj)
    errs = []
    for k in range(3):
        e, e32 = rel(g16[k], g64[k]), rel(g32[k], g64[k])
        print(f"VTI precision {precision} grad[{k}]: vs fp64 {e:.3e} (FP32 full storage {e32:.3e})")
        errs.append(e)
    assert max(errs) < BOUND[precision]
