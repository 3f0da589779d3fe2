"""GPU parity against the CPU oracle (the reference's own sources, built in
oracle/_ref): traces within 1e-5 relative L2 of the FP32 build, gradients
within 1e-4, on seeded inputs; the FP64 build's distance is reported."""
import numpy as np
import pytest

from fwi3d_b200 import ops, synth

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5
GRAD_TOL = 1e-4


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _acoustic(n=32, steps=200):
    return synth.acoustic_linear(n=n, nsteps=steps, taper=6, rec_stride=3)


def _elastic(n=28, steps=160, mt=True):
    sv = synth.elastic_layered(n=n, nsteps=steps, taper=6, rec_stride=3, nshots=1)
    sv.par.sxyz = [[0.5 * n * sv.dx, 0.4 * n * sv.dx, 0.3 * n * sv.dx]]
    sv.par.mt = mt
    return sv


def _vti(n=28, steps=160):
    sv = synth.vti_layered(nx=n, ny=n + 4, nz=n - 2, nsteps=steps, taper=6, rec_stride=3, nshots=1, dt=0.0005)
    sv.par.sxyz = [[0.5 * n * sv.dx, 0.4 * n * sv.dx, 0.3 * n * sv.dx]]
    return sv


BCS = [(1, 2, 2, 2, 2, 2), (2, 2, 2, 2, 2, 2), (1, 1, 1, 1, 1, 1), (2, 1, 3, 2, 1, 2)]


@pytest.mark.parametrize("bc", BCS)
def test_acoustic_traces(oracle_fp32, bc):
    sv = _acoustic()
    sv.par.set_bc(*bc)
    d = ops.from_survey(sv).forward(False, sv.model)
    ref, info = oracle_fp32.modeling(sv, precision="fp32")
    assert rel(d, ref) < TRACE_TOL


@pytest.mark.parametrize("mt", [True, False])
@pytest.mark.parametrize("bc", [(1, 2, 2, 2, 2, 2), (2, 1, 2, 1, 2, 1)])
def test_elastic_traces(oracle_fp32, mt, bc):
    sv = _elastic(mt=mt)
    sv.par.set_bc(*bc)
    d = ops.from_survey(sv).forward(False, sv.model)
    ref, _ = oracle_fp32.modeling(sv, precision="fp32")
    assert rel(d, ref) < TRACE_TOL


@pytest.mark.parametrize("bc", [(1, 2, 2, 2, 2, 2), (2, 1, 2, 1, 2, 1)])
def test_vti_traces(oracle_fp32, bc):
    sv = _vti()
    sv.par.set_bc(*bc)
    d = ops.from_survey(sv).forward(False, sv.model)
    ref, _ = oracle_fp32.modeling(sv, precision="fp32")
    assert rel(d, ref) < TRACE_TOL


def _grad_case(oracle, sv, sub, trace_tol=TRACE_TOL):
    sv.par.sub = sub
    rng = np.random.default_rng(0)
    ref, _ = oracle.modeling(sv, precision="fp32")
    adj = (rng.standard_normal(ref.shape) * np.abs(ref).max()).astype(np.float32)
    op = ops.from_survey(sv)
    syn = op.forward(False, sv.model)
    g = op.jacobianT(False, None, sv.model, adj)
    s32, g32, _ = oracle.forward_jacobianT(sv, adj, precision="fp32")
    assert rel(syn, s32) < trace_tol
    for k in range(g32.shape[0]):
        assert rel(g[k], g32[k]) < GRAD_TOL, f"parameter {k}"


@pytest.mark.parametrize("sub", [1, 4])
def test_acoustic_gradient(oracle_fp32, sub):
    _grad_case(oracle_fp32, _acoustic(n=28, steps=151), sub)


@pytest.mark.parametrize("mt", [True, False])
def test_elastic_gradient(oracle_fp32, mt):
    _grad_case(oracle_fp32, _elastic(n=26, steps=150, mt=mt), 1)


def test_vti_gradient(oracle_fp32):
    _grad_case(oracle_fp32, _vti(n=26, steps=151), 3)


def test_config1_full_size(oracle_fp32):
    """Acoustic 101^3 x 1000 steps (config 1) against both oracle builds."""
    sv = synth.acoustic_linear()
    d = ops.from_survey(sv).forward(False, sv.model)
    ref32, _ = oracle_fp32.modeling(sv, precision="fp32")
    ref64, _ = oracle_fp32.modeling(sv, precision="fp64")
    e32, e64 = rel(d, ref32), rel(d, ref64)
    print(f"config1: vs fp32 {e32:.3e}  vs fp64 {e64:.3e}  fp32-vs-fp64 {rel(ref32, ref64):.3e}")
    assert e32 < TRACE_TOL


def test_batch_matches_single_shot_operator():
    """Shots batched in one launch give the traces of separate operators."""
    sv = synth.elastic_layered(n=28, nsteps=120, taper=6, rec_stride=4, nshots=3)
    for s in range(3):
        sv.par.sxyz[s] = [(0.3 + 0.2 * s) * 28 * sv.dx, (0.5 - 0.1 * s) * 28 * sv.dx, 0.2 * 28 * sv.dx]
    batch = ops.forward_batch(sv)
    for s in range(3):
        single = ops.from_survey(sv, s).forward(False, sv.model)
        assert rel(batch[s], single) < 1e-6


# --- grids large enough for the fused interior kernel (nz >= 32, nx >= 16, ny > 16) ---

def _elastic_fused(mt=True):
    sv = synth.elastic_layered(n=48, nsteps=150, taper=6, rec_stride=3, nshots=1)
    # non-cubic grid so that tiles, chunks and closures all differ per axis
    sv.model = np.ascontiguousarray(sv.model[:, :36, :40, :48])
    sv.nx, sv.ny, sv.nz = 40, 36, 48
    sv.par.sxyz = [[0.5 * 40 * sv.dx, 0.45 * 36 * sv.dx, 0.3 * 48 * sv.dx]]
    sv.par.rxyz = [[r for r in sv.par.rxyz[0] if r[0] <= 39 * sv.dx and r[1] <= 35 * sv.dx]]
    sv.par.mt = mt
    return sv


def _vti_fused():
    sv = synth.vti_layered(nx=40, ny=36, nz=48, nsteps=150, taper=6, rec_stride=3, nshots=1, dt=0.0005)
    sv.par.sxyz = [[0.5 * 40 * sv.dx, 0.45 * 36 * sv.dx, 0.3 * 48 * sv.dx]]
    return sv


@pytest.mark.parametrize("mt", [True, False])
def test_elastic_fused_traces(oracle_fp32, mt):
    sv = _elastic_fused(mt)
    d = ops.from_survey(sv).forward(False, sv.model)
    ref, _ = oracle_fp32.modeling(sv, precision="fp32")
    assert rel(d, ref) < TRACE_TOL


def test_vti_fused_traces(oracle_fp32):
    sv = _vti_fused()
    d = ops.from_survey(sv).forward(False, sv.model)
    ref, _ = oracle_fp32.modeling(sv, precision="fp32")
    assert rel(d, ref) < TRACE_TOL


def test_fused_matches_per_point(monkeypatch):
    """The marching kernel (default), the interior fused kernel (FWI_MARCH=0)
    and the per-point kernels (FWI_MARCH=0 FWI_FUSED=0) agree to rounding."""
    out = {}
    for tag, march, fused in (("p", "0", "0"), ("f", "0", "1"), ("m", "1", "1")):
        monkeypatch.setenv("FWI_MARCH", march)
        monkeypatch.setenv("FWI_FUSED", fused)
        for name, sv in (("e", _elastic_fused()), ("v", _vti_fused())):
            out[name + tag] = ops.from_survey(sv).forward(False, sv.model)
    for name in "ev":
        assert rel(out[name + "f"], out[name + "p"]) < 2e-6
        assert rel(out[name + "m"], out[name + "p"]) < 2e-6


def test_fused_plane_copies(monkeypatch):
    """The fused kernel's bulk-tensor plane copies (nz % 4 == 0) give the same
    bits as its per-thread copies (FWI_TMA=0); a grid with nz % 4 != 0 takes
    the per-thread copies and matches the per-point kernels."""
    for name, sv in (("e", _elastic_fused()), ("v", _vti_fused())):
        monkeypatch.setenv("FWI_TMA", "1")
        t = ops.from_survey(sv).forward(False, sv.model)
        monkeypatch.setenv("FWI_TMA", "0")
        a = ops.from_survey(sv).forward(False, sv.model)
        assert np.array_equal(t, a), name
    monkeypatch.delenv("FWI_TMA")
    sv = _elastic_fused()
    sv.model = np.ascontiguousarray(sv.model[:, :, :, :46])
    sv.nz = 46
    f = ops.from_survey(sv).forward(False, sv.model)
    monkeypatch.setenv("FWI_FUSED", "0")
    p = ops.from_survey(sv).forward(False, sv.model)
    assert rel(f, p) < 2e-6


def test_march_chunks_and_batch(monkeypatch):
    """Marching kernel with several y chunks per tile column and a batch of
    shots against the per-point kernels."""
    sv = synth.elastic_layered(n=64, nsteps=100, taper=6, rec_stride=4, nshots=3)
    for s in range(3):
        sv.par.sxyz[s] = [(0.3 + 0.2 * s) * 64 * sv.dx, (0.5 - 0.1 * s) * 64 * sv.dx, 0.2 * 64 * sv.dx]
    sv.par.set_bc(2, 1, 2, 1, 2, 1)
    monkeypatch.setenv("FWI_MARCH", "1")
    m = ops.forward_batch(sv)
    monkeypatch.setenv("FWI_MARCH", "0")
    monkeypatch.setenv("FWI_FUSED", "0")
    p = ops.forward_batch(sv)
    assert rel(m, p) < 2e-6


def test_elastic_fused_gradient(oracle_fp32):
    _grad_case(oracle_fp32, _elastic_fused(True), 1)


def _das(n=28, steps=140, mt=True):
    """Elastic survey recorded by DAS channels (gauge length 30 m) along
    fibres of mixed dip and azimuth, away from the edges."""
    sv = _elastic(n=n, steps=steps, mt=mt)
    rng = np.random.default_rng(4)
    rec = []
    for k in range(40):
        x, y = rng.uniform(0.25, 0.75, 2) * (n - 1) * sv.dx
        z = rng.uniform(0.2, 0.6) * (n - 1) * sv.dx
        rec.append([float(x), float(y), float(z), float(rng.uniform(-1.2, 1.2)), float(rng.uniform(0, 6.28))])
    sv.par.rxyz = [rec]
    sv.par.gl = 0.03
    return sv


def _das_tol(oracle, sv):
    """A DAS channel records the difference of two nearby samples divided by
    the gauge length, so FP32 cancellation is at the 1e-5 level: the
    reference's own FP32 build is 0.9e-5 to 1.3e-5 from its FP64 build on these
    cases.  Traces are held to twice that distance (at least 1e-5)."""
    r32, _ = oracle.modeling(sv, precision="fp32")
    r64, _ = oracle.modeling(sv, precision="fp64")
    return max(TRACE_TOL, 2 * rel(r32, r64)), r32, r64


@pytest.mark.parametrize("seismotype", [0, 1])
def test_das_traces(oracle_fp32, seismotype):
    sv = _das()
    sv.par.seismotype = seismotype
    d = ops.from_survey(sv).forward(False, sv.model)
    tol, ref, ref64 = _das_tol(oracle_fp32, sv)
    assert d.shape[0] == 1
    assert rel(d, ref) < tol
    assert rel(d, ref64) < tol


def test_das_gradient(oracle_fp32):
    sv = _das(n=26, steps=120)
    tol, _, _ = _das_tol(oracle_fp32, sv)
    _grad_case(oracle_fp32, sv, 1, trace_tol=tol)


@pytest.mark.parametrize("bc", [(1, 2, 2, 2, 2, 2), (2, 1, 3, 2, 1, 2)])
def test_acoustic_fused_traces(oracle_fp32, bc, monkeypatch):
    """The acoustic marching kernel (grids with nz >= 38, nx >= 22) against the
    oracle and against the per-point kernel (FWI_FUSED=0)."""
    sv = synth.acoustic_linear(n=44, nsteps=150, taper=6, rec_stride=3)
    sv.par.set_bc(*bc)
    monkeypatch.setenv("FWI_FUSED", "1")  # the marching kernel also below its size threshold
    d = ops.from_survey(sv).forward(False, sv.model)
    ref, _ = oracle_fp32.modeling(sv, precision="fp32")
    assert rel(d, ref) < TRACE_TOL
    monkeypatch.setenv("FWI_FUSED", "0")
    d0 = ops.from_survey(sv).forward(False, sv.model)
    assert rel(d, d0) < 2e-6


def test_acoustic_fused_gradient(oracle_fp32, monkeypatch):
    monkeypatch.setenv("FWI_FUSED", "1")
    _grad_case(oracle_fp32, synth.acoustic_linear(n=40, nsteps=120, taper=5, rec_stride=3), 1)


def test_graph_replay_matches_plain_launches(monkeypatch):
    """Modeling runs replayed as three-step CUDA graphs (default) give the
    traces of plain launches (FWI_GRAPHS=0) bit for bit, for a batch run in
    uneven chunks (the serving loop's pattern) and for a whole-axis run."""
    from fwi3d_b200 import _lib
    import ctypes as C

    sv = _elastic_fused()
    out = {}
    for g in ("1", "0"):
        monkeypatch.setenv("FWI_GRAPHS", g)
        out["op" + g] = ops.from_survey(sv).forward(False, sv.model)
        lib = _lib.load()
        dom = ops.Domain(sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.nmodels)
        w = np.ascontiguousarray(sv.wavelet, dtype=np.float32)
        sx = np.ascontiguousarray(np.asarray(sv.par.sxyz, dtype=np.float32))
        rx = np.ascontiguousarray(np.asarray(sv.par.rxyz, dtype=np.float32))
        h = C.c_void_p()
        _lib.check(lib.fwi_batch_create(C.byref(h), 0, C.byref(dom.grid()), sv.nmodels,
                                        C.byref(ops.to_cparam(sv.par)),
                                        _lib.fptr(np.ascontiguousarray(sv.model, dtype=np.float32)), _lib.fptr(w),
                                        1, w.shape[-1], sv.dt_data, 1, _lib.fptr(sx), rx.shape[1], _lib.fptr(rx)))
        info = _lib.OpInfo()
        _lib.check(lib.fwi_batch_get_info(h, C.byref(info), None))
        _lib.check(lib.fwi_batch_reset(h))
        left = info.nt - 1
        for k in (1, 7, 20, 2, 50):
            _lib.check(lib.fwi_batch_run(h, min(k, left)))
            left -= min(k, left)
        _lib.check(lib.fwi_batch_run(h, left))
        tr = np.zeros((1, info.nrcomp, rx.shape[1], w.shape[-1]), dtype=np.float32)
        _lib.check(lib.fwi_batch_traces(h, _lib.fptr(tr)))
        lib.fwi_batch_destroy(h)
        out["b" + g] = tr
    assert np.array_equal(out["op1"], out["op0"])
    assert np.array_equal(out["b1"], out["b0"])


def test_das_batch_equals_operator():
    """DAS channels on the batch path (two shots in one launch, strain formed
    on the device) against the operator path shot by shot."""
    sv = _das(n=28, steps=120)
    n = 28
    sv.par.sxyz = [[0.5 * n * sv.dx, 0.4 * n * sv.dx, 0.3 * n * sv.dx], [0.4 * n * sv.dx, 0.55 * n * sv.dx, 0.25 * n * sv.dx]]
    sv.par.rxyz = [sv.par.rxyz[0], sv.par.rxyz[0]]
    sv.par.ns = 2
    d = ops.forward_batch(sv)
    assert d.shape[1] == 1
    for s in range(2):
        ref = ops.from_survey(sv, s).forward(False, sv.model)
        assert rel(d[s], ref) < 1e-6, s


def test_das_objective_matches_reference(oracle_fp32):
    """The device FWI objective with DAS channels (strain on the device, its
    adjoint spread back to the dipoles) against nlls_fwi of the reference's
    FP32 build; the host residual path (FWI_HOST_RESIDUAL=1) gives the same."""
    import os

    sv = _das(n=26, steps=120)
    sv.par.sub = 1
    tol, _, _ = _das_tol(oracle_fp32, sv)
    true = synth.Survey(sv.name, sv.nmodels, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.model * np.float32(1.02),
                        sv.wavelet, sv.dt_data, sv.par.copy())
    obs = oracle_fp32.modeling(true, precision="fp32")[0][None].astype(np.float32)
    ref = oracle_fp32.fwi(sv, obs, solver="none")
    f, g = ops.FwiObjective(sv, obs, normalize=True, batch=1).evaluate(sv.model)
    assert abs(f - ref["f"][0]) / ref["f"][0] < 10 * tol
    for k in range(3):
        assert rel(g[k], ref["grad"][k]) < 1e-4 + 10 * tol, k
    os.environ["FWI_HOST_RESIDUAL"] = "1"
    try:
        fh, gh = ops.FwiObjective(sv, obs, normalize=True, batch=1).evaluate(sv.model)
    finally:
        del os.environ["FWI_HOST_RESIDUAL"]
    assert fh == pytest.approx(f, rel=1e-6)
    assert rel(gh, g) < 1e-6


@pytest.mark.parametrize("case", ["elastic_velocity", "acoustic", "das"])
def test_device_trace_output_equals_host(case, monkeypatch):
    """Batch traces post-processed on the device (Dt for velocity data,
    dt/dt_data, sinc resampling to the data axis) equal the host formulation
    (FWI_HOST_OUTPUT=1) bit for bit, for a whole batch and for shot slots."""
    if case == "acoustic":
        sv = synth.acoustic_linear(n=30, nsteps=90, taper=4, rec_stride=3)
    elif case == "das":
        sv = _das(n=28, steps=90)
    else:
        sv = _elastic(n=28, steps=90)
        sv.par.seismotype = 1
    dev = ops.forward_batch(sv)
    monkeypatch.setenv("FWI_HOST_OUTPUT", "1")
    host = ops.forward_batch(sv)
    assert np.array_equal(dev, host)
