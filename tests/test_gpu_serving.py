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
