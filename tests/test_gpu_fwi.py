"""FWI objective, FP16 snapshot storage, finite-difference check, l-BFGS and
the torch.autograd wrapper on the GPU."""
import numpy as np
import pytest

from fwi3d_b200 import ops, synth

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _problem(n=28, steps=120, nside=2, storage=0):
    sv = synth.elastic_anomaly(n=n, nsteps=steps, nshots_side=nside, taper=6, rec_stride=3)
    sv.par.sub = 1
    sv.par.snapshot_storage = storage
    true = synth.Survey(sv.name, sv.nmodels, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz,
                        sv.extra["true_model"], sv.wavelet, sv.dt_data, sv.par.copy())
    obs = ops.forward_batch(true)
    return sv, obs


def _ht(r, dt):
    """Trapezoid weights of the time axis (misc.cpp:44-56)."""
    a = (r * np.float32(dt)).astype(np.float32)
    a[..., 0] = (r[..., 0].astype(np.float64) * 0.5 * dt).astype(np.float32)
    a[..., -1] = (r[..., -1].astype(np.float64) * 0.5 * dt).astype(np.float32)
    return a


def test_objective_matches_per_shot_operators():
    sv, obs = _problem()
    obj = ops.FwiObjective(sv, obs, normalize=True, batch=4)
    f, g, r = obj.evaluate(sv.model, want_residual=True)
    syn = ops.forward_batch(sv)
    assert rel(r, syn - obs) < 1e-6
    dt = sv.dt_data
    rr = (syn - obs).astype(np.float64)
    dnorm = float(np.sum(obs.astype(np.float64) ** 2)) * dt
    fref = 0.5 * dt * (np.sum(rr ** 2) - 0.5 * np.sum(rr[..., 0] ** 2 + rr[..., -1] ** 2)) / dnorm
    assert abs(f - fref) / fref < 1e-6
    gsum = np.zeros_like(g, dtype=np.float64)
    for s in range(len(sv.par.sxyz)):
        op = ops.from_survey(sv, s)
        op.forward(False, sv.model)
        gsum += op.jacobianT(False, None, sv.model, _ht(r[s], dt))
        op.close()
    gsum /= dnorm
    for k in range(3):
        assert rel(g[k], gsum[k]) < 1e-5, k


def test_objective_batch_size_invariant():
    sv, obs = _problem()
    f4, g4 = ops.FwiObjective(sv, obs, batch=4).evaluate(sv.model)
    f1, g1 = ops.FwiObjective(sv, obs, batch=1).evaluate(sv.model)
    f3, g3 = ops.FwiObjective(sv, obs, batch=3).evaluate(sv.model)
    assert abs(f1 - f4) / f4 < 1e-6 and abs(f3 - f4) / f4 < 1e-6
    assert rel(g1, g4) < 1e-6 and rel(g3, g4) < 1e-6


def test_fp16_snapshots_gradient_error():
    """FP16 second-difference snapshot storage: gradient within 1e-4 of the
    FP32-storage gradient (half the snapshot memory)."""
    sv, obs = _problem()
    o32 = ops.FwiObjective(sv, obs, batch=4)
    f32, g32 = o32.evaluate(sv.model)
    sv.par.snapshot_storage = 1
    o16 = ops.FwiObjective(sv, obs, batch=4)
    f16, g16 = o16.evaluate(sv.model)
    assert f16 == pytest.approx(f32, rel=1e-6)
    for k in range(3):
        assert rel(g16[k], g32[k]) < 1e-4, k
    assert o16.device_bytes() < 0.75 * o32.device_bytes()


def test_fp16_snapshots_vs_fp64_oracle(oracle_fp32):
    """Single-shot operator gradient with FP16 storage against the reference's
    FP64 build: relative L2 error at most 1e-3 per parameter."""
    sv = synth.elastic_layered(n=26, nsteps=150, taper=6, rec_stride=3, nshots=1)
    sv.par.sxyz = [[0.5 * 26 * sv.dx, 0.4 * 26 * sv.dx, 0.3 * 26 * sv.dx]]
    sv.par.sub = 1
    rng = np.random.default_rng(0)
    ref, _ = oracle_fp32.modeling(sv, precision="fp32")
    adj = (rng.standard_normal(ref.shape) * np.abs(ref).max()).astype(np.float32)
    _, g64, _ = oracle_fp32.forward_jacobianT(sv, adj, precision="fp64")
    sv.par.snapshot_storage = 1
    op = ops.from_survey(sv)
    op.forward(False, sv.model)
    g = op.jacobianT(False, None, sv.model, adj)
    for k in range(3):
        assert rel(g[k], g64[k]) < 1e-3, k


def test_finite_difference_directional_derivative():
    """(f(m + e dm) - f(m - e dm)) / 2e against <g, dm> for e = 1e-2 .. 1e-4."""
    sv, obs = _problem()
    obj = ops.FwiObjective(sv, obs, batch=4)
    m = sv.model.astype(np.float32)
    f0, g = obj.evaluate(m)
    rng = np.random.default_rng(3)
    from scipy.ndimage import gaussian_filter

    dm = np.stack([gaussian_filter(rng.standard_normal(m.shape[1:]), 3.0) for _ in range(3)])
    dm = (dm / np.abs(dm).max() * 0.02 * m).astype(np.float64)  # 2 % of the model at e = 1
    dm[:, :, :, :3] = 0.0  # keep the surface layer (sources, receivers) fixed
    gd = float(np.sum(g.astype(np.float64) * dm))
    errs = []
    for e in (1e-1, 3e-2, 1e-2):
        fp, _ = obj.evaluate((m + e * dm).astype(np.float32))
        fm, _ = obj.evaluate((m - e * dm).astype(np.float32))
        errs.append(abs((fp - fm) / (2 * e) - gd) / abs(gd))
    print("FD relative errors", errs)
    assert min(errs) < 0.05, errs


def test_lbfgs_decreases_misfit():
    """Two l-BFGS iterations with the regular Wolfe search on the device
    objective: the misfit decreases at each accepted step."""
    from fwi3d_b200 import nlsolver

    sv, obs = _problem()
    obj = ops.FwiObjective(sv, obs, batch=4)
    prob = nlsolver.Problem(sv.model.astype(np.float32), obj.evaluate, nlsolver.Backend("cuda:0"))
    s = nlsolver.Lbfgs(2, max_trial=10, ls=nlsolver.RegularWolfe())
    s.run(prob)
    assert len(s.func) == 3
    assert s.func[2] < s.func[1] < s.func[0]


def test_autograd_function_gradient():
    import torch

    from fwi3d_b200 import autograd

    sv, obs = _problem()
    obj = ops.FwiObjective(sv, obs, batch=4)
    f0, g0 = obj.evaluate(sv.model)
    mt = torch.tensor(sv.model, device="cuda:0", requires_grad=True)
    f = autograd.misfit(mt, obj)
    f.backward()
    assert float(f) == pytest.approx(f0, rel=1e-12)
    assert rel(mt.grad.cpu().numpy()[:3], g0) < 1e-7


def test_checkpointed_gradient_matches_full_storage():
    """Under an HBM budget below full storage the forward keeps checkpoints and
    the adjoint recomputes segments: same misfit and gradient, less memory."""
    sv, obs = _problem()
    full = ops.FwiObjective(sv, obs, batch=4)
    f0, g0 = full.evaluate(sv.model)
    sv.par.snapshot_budget_gb = 0.06
    ck = ops.FwiObjective(sv, obs, batch=4)
    f1, g1 = ck.evaluate(sv.model)
    assert f1 == pytest.approx(f0, rel=1e-7)
    assert rel(g1, g0) < 1e-6
    assert ck.device_bytes() < 0.6 * full.device_bytes()
    sv.par.snapshot_budget_gb = 0.001  # below the checkpointing minimum: a clear error
    with pytest.raises(Exception, match="snapshot budget"):
        ops.FwiObjective(sv, obs, batch=4).evaluate(sv.model)


def test_sharded_objective_matches_single_process():
    """Shots split over two ranks (rank-strided) and summed as the all-reduce
    does: same misfit and gradient as one objective over all shots."""
    from fwi3d_b200 import distributed

    sv, obs = _problem()
    f, g = ops.FwiObjective(sv, obs, normalize=True, batch=4).evaluate(sv.model)
    one = distributed.ShardedObjective(sv, obs, rank=0, world=1, batch=4)
    f1, g1 = one.evaluate(sv.model)
    assert f1 == pytest.approx(f, rel=1e-9) and rel(g1, g) < 1e-7
    parts = [distributed.ShardedObjective(sv, obs, rank=r, world=2, batch=2) for r in range(2)]
    fs, gs, dns = 0.0, 0.0, 0.0
    for p in parts:
        fl, gl = p.obj.evaluate(sv.model)
        fs, gs, dns = fs + fl, gs + gl.astype(np.float64), dns + p.dn_local
    assert fs / dns == pytest.approx(f, rel=1e-6)
    assert rel(gs / dns, g) < 1e-6


@pytest.mark.parametrize("seismotype", [0, 1])
def test_device_residual_matches_host_path(monkeypatch, seismotype):
    """The objective's residual on the device (default: sinc resampling,
    misfit partials, Ht, time reversal, Dt for velocity data) gives the host
    path's residual bit for bit (FWI_HOST_RESIDUAL=1), its misfit to FP64
    reassociation, and its gradient up to the order of the adjoint
    injection's atomic additions."""
    sv, obs = _problem(nside=2)
    sv.par.seismotype = seismotype
    out = {}
    for tag, env in (("host", "1"), ("dev", "0")):
        monkeypatch.setenv("FWI_HOST_RESIDUAL", env)
        obj = ops.FwiObjective(sv, obs, batch=2)
        out[tag] = obj.evaluate(sv.model, want_residual=True)
        obj.close()
    fh, gh, rh = out["host"]
    fd, gd, rd = out["dev"]
    assert np.array_equal(rh, rd)
    assert abs(fd - fh) <= 1e-12 * abs(fh)
    assert rel(gd, gh) < 1e-6
