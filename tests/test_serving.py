"""Serving loop host logic with a fake executor and a simulated clock:
admission by memory budget, batching of compatible shots, continuous
admission of late arrivals, latency bookkeeping."""
import numpy as np

from fwi3d_b200 import serving, synth


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-4)


class FakeExecutor:
    """Each advanced step of a session costs 1 ms of simulated time."""

    def __init__(self, clock, free=10 ** 12):
        self.clock, self.free = clock, free
        self.open_sessions = []
        self.max_shots = 0
        self.log = []

    def free_bytes(self):
        return self.free

    def open_batch(self, reqs, model):
        s = {"left": reqs[0].survey.nt_data - 1, "points": 1000, "ns": len(reqs), "ids": [r.rid for r in reqs]}
        self.open_sessions.append(s)
        self.max_shots = max(self.max_shots, len(reqs))
        self.log.append(("open", self.clock.t, tuple(s["ids"])))
        return s

    def advance(self, s, n):
        k = min(n, s["left"])
        s["left"] -= k
        self.clock.t += 1e-3 * k / max(1, len(self.open_sessions))
        return k

    def wait(self, s):
        pass

    def finish(self, s):
        self.open_sessions.remove(s)
        self.log.append(("done", self.clock.t, tuple(s["ids"])))
        return [np.full(3, r, dtype=np.float32) for r in s["ids"]]

    def gradient(self, req, model):
        return (1.0, np.zeros(3))


def _req(rid, model_id="m", steps=100, arrival=0.0, n=24, mode="modeling"):
    sv = synth.elastic_layered(n=n, nsteps=steps, taper=4, rec_stride=6, nshots=1)
    return serving.Request(rid, model_id, mode, sv, arrival=arrival)


def test_compatible_shots_are_batched():
    clk = FakeClock()
    ex = FakeExecutor(clk)
    reqs = [_req(i) for i in range(5)] + [_req(9, model_id="other")]
    srv = serving.Server({"m": None, "other": None}, executor=ex, chunk=10, max_batch=4)
    rep = srv.run(reqs, clock=clk, sleep=clk.sleep)
    assert all(r.done is not None for r in reqs)
    assert ex.max_shots == 4
    opens = [e for e in ex.log if e[0] == "open"]
    assert len(opens) == 3  # 4 + 1 on model m, 1 on model other
    assert rep.summary()["p99_s"] >= rep.summary()["p50_s"] >= 0


def test_budget_limits_admission():
    clk = FakeClock()
    ex = FakeExecutor(clk)
    reqs = [_req(i) for i in range(4)]
    one = serving.session_bytes(reqs[0].survey, 1)
    srv = serving.Server({"m": None}, executor=ex, chunk=10, max_batch=8, budget_bytes=int(2.5 * one))
    srv.run(reqs, clock=clk, sleep=clk.sleep)
    assert ex.max_shots == 2  # three shots do not fit the budget
    assert all(r.done is not None for r in reqs)


def test_late_arrival_is_admitted_while_others_run():
    clk = FakeClock()
    ex = FakeExecutor(clk)
    long = _req(0, steps=400)
    late = _req(1, model_id="x", steps=50, arrival=0.05)
    srv = serving.Server({"m": None, "x": None}, executor=ex, chunk=10)
    srv.run([long, late], clock=clk, sleep=clk.sleep)
    assert late.admitted < long.done  # joined while the long session was running
    assert late.done < long.done
    assert late.done - late.arrival < long.done - long.arrival


def test_session_bytes_grow_with_shots_and_gradient():
    sv = synth.elastic_layered(n=24, nsteps=50, taper=4, rec_stride=6, nshots=1)
    assert serving.session_bytes(sv, 2) > serving.session_bytes(sv, 1)
    assert serving.session_bytes(sv, 1, gradient=True) > serving.session_bytes(sv, 1)
