"""Serving loop on the GPU: a small mix of modeling and gradient shots of all
three physics arriving over time; every result equals the same request run
alone (relative L2 within 1e-6)."""
import numpy as np
import pytest

from fwi3d_b200 import ops, servemix, serving

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(np.asarray(b, np.float64)), 1e-30))


def test_mix_results_equal_alone():
    models, reqs = servemix.make_mix(nreq=10, rate=40.0, seed=11, grids=((40, 40, 40), (48, 44, 40)),
                                     steps=(60, 80), rec=(8,), p_gradient=0.3)
    srv = serving.Server(models, chunk=20, max_batch=4)
    rep = srv.run(reqs)
    s = rep.summary()
    assert s["requests"] == len(reqs) and s["p99_s"] >= s["p50_s"] > 0
    assert any(r.mode == "gradient" for r in reqs) and any(r.mode == "modeling" for r in reqs)
    for r in reqs:
        assert r.done is not None and r.done >= r.arrival
        if r.mode == "modeling":
            alone = ops.forward_batch(r.survey)[0]
            assert rel(r.result, alone) < 1e-6, r.rid
        else:
            obj = ops.FwiObjective(r.survey, r.observed, normalize=True, batch=1)
            f, g = obj.evaluate(models[r.model_id])
            assert r.result[0] == pytest.approx(f, rel=1e-6)
            assert rel(r.result[1], g) < 1e-6, r.rid


def _shot(req, sx, rid=None):
    """The request's survey with another source position (same key)."""
    sv = req.survey
    par = sv.par.copy()
    par.sxyz = [list(sx)]
    s2 = type(sv)(f"{sv.name}_s", sv.nmodels, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.model, sv.wavelet,
                  sv.dt_data, par)
    return serving.Request(req.rid * 10 + 1 if rid is None else rid, req.model_id, req.mode, s2,
                           observed=req.observed)


def _mix(mode, seed=3):
    models, reqs = servemix.make_mix(nreq=1, rate=40.0, seed=seed, grids=((44, 40, 36),), steps=(60,), rec=(8,),
                                     p_gradient=1.0 if mode == "gradient" else 0.0)
    return models, reqs[0]


def test_slots_join_a_running_session_and_match_alone():
    """A session of two slots: shot A from step 0, B joins the idle slot 20
    steps later, C takes A's slot when A completes; the three data sets equal
    each shot run alone (the step is per shot; only the start differs)."""
    models, a = _mix("modeling")
    sv = a.survey
    b = _shot(a, [0.6 * (sv.nx - 1) * sv.dx, 0.45 * (sv.ny - 1) * sv.dy, 0.02])
    c = _shot(a, [0.35 * (sv.nx - 1) * sv.dx, 0.55 * (sv.ny - 1) * sv.dy, 0.02], rid=99)
    ex = serving.GpuExecutor()
    s = ex.open_batch([a], models[a.model_id], slots=2)
    try:
        ex.advance(s, 20)
        assert ex.join(s, 1, b)
        ex.advance(s, ex.remaining(s, 0))
        assert ex.remaining(s, 0) == 0 and ex.remaining(s, 1) == 20
        da = ex.finish_slot(s, 0)
        assert ex.join(s, 0, c)
        ex.advance(s, ex.remaining(s, 1))
        db = ex.finish_slot(s, 1)
        ex.advance(s, ex.remaining(s, 0))
        dc = ex.finish_slot(s, 0)
    finally:
        ex.close(s)
    for req, d in ((a, da), (b, db), (c, dc)):
        alone = ops.forward_batch(req.survey)[0]
        assert rel(d, alone) < 1e-6, req.rid


def test_join_refuses_a_source_in_a_taper_zone():
    models, r0 = _mix("modeling")
    sv = r0.survey
    edge = _shot(r0, [2 * sv.dx, 0.5 * (sv.ny - 1) * sv.dy, 0.02])  # inside the 10-point x taper
    ex = serving.GpuExecutor()
    s = ex.open_batch([r0], models[r0.model_id], slots=2)
    try:
        assert not ex.join(s, 1, edge)
        ex.advance(s, ex.remaining(s, 0))
        d = ex.finish_slot(s, 0)
    finally:
        ex.close(s)
    assert rel(d, ops.forward_batch(r0.survey)[0]) < 1e-6


def _alone(req, model):
    obj = ops.FwiObjective(req.survey, req.observed, normalize=True, batch=1)
    try:
        return obj.evaluate(model)
    finally:
        obj.close()


def test_batched_gradient_requests_match_alone():
    """Three gradient requests of one key in one evaluation (one objective per
    shot from the same launches), then two other requests through the kept
    objective of that batch size: each equals the request evaluated alone."""
    models, r0 = _mix("gradient", seed=4)
    sv = r0.survey
    pos = [(0.3, 0.6), (0.62, 0.4), (0.45, 0.3), (0.55, 0.62), (0.38, 0.45)]
    rs = [_shot(r0, [px * (sv.nx - 1) * sv.dx, py * (sv.ny - 1) * sv.dy, 0.02], rid=k) for k, (px, py) in enumerate(pos)]
    model = models[r0.model_id]
    ex = serving.GpuExecutor()
    try:
        out = ex.gradients(rs[:3], model)
        assert ex.cached_bytes() > 0
        out2 = ex.gradients(rs[3:], model)
    finally:
        ex.drop_cache()
    assert ex.cached_bytes() == 0
    for r, (f1, g1) in zip(rs, out + out2):
        f, g = _alone(r, model)
        assert f1 == pytest.approx(f, rel=1e-6), r.rid
        assert rel(g1, g) < 1e-6, r.rid


def test_kept_gradient_objective_matches_a_fresh_one():
    models, r0 = _mix("gradient", seed=4)
    sv = r0.survey
    r1 = _shot(r0, [0.3 * (sv.nx - 1) * sv.dx, 0.6 * (sv.ny - 1) * sv.dy, 0.02])
    model = models[r0.model_id]
    ex = serving.GpuExecutor()
    try:
        ex.gradients([r0], model)
        (f1, g1), = ex.gradients([r1], model)   # the kept objective with r1's shot
    finally:
        ex.drop_cache()
    f, g = _alone(r1, model)
    assert f1 == pytest.approx(f, rel=1e-9)
    assert rel(g1, g) < 1e-9
