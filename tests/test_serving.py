"""Serving loop host logic with a fake executor and a simulated clock:
admission by memory budget, batching of compatible shots, continuous
admission of late arrivals, shots joining a running session's free slots,
gradient requests of one key evaluated together, the gradient objectives
kept between requests, latency bookkeeping."""
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
    """Each advanced step of a session costs 1 ms of simulated time (shared
    by the open sessions).  Slots follow the C ABI: a slot's shot is done
    nt steps after its start."""

    def __init__(self, clock, free=10 ** 12, refuse=(), gradient_bytes=0):
        self.clock, self.free = clock, free
        self.refuse = set(refuse)
        self.open_sessions = []
        self.max_shots = 0
        self.log = []
        self.cache = 0
        self.gradient_bytes = gradient_bytes
        self.drops = 0
        self.grad_batches = []

    def free_bytes(self):
        return self.free

    def open_batch(self, reqs, model, slots=None):
        nt = reqs[0].survey.nt_data
        n = max(len(reqs), slots or 0)
        s = {"nt": nt, "it": 0, "t0": [0] * len(reqs) + [-nt] * (n - len(reqs)), "points": 1000,
             "ids": [r.rid for r in reqs] + [None] * (n - len(reqs))}
        self.open_sessions.append(s)
        self.max_shots = max(self.max_shots, len(reqs))
        self.log.append(("open", self.clock.t, tuple(s["ids"])))
        return s

    def advance(self, s, n):
        s["it"] += n
        self.clock.t += 1e-3 * n / max(1, len(self.open_sessions))
        return n

    def wait(self, s):
        pass

    def remaining(self, s, slot):
        return max(0, s["t0"][slot] + s["nt"] - s["it"])

    def join(self, s, slot, req):
        if req.rid in self.refuse:
            return False
        assert self.remaining(s, slot) == 0
        s["t0"][slot] = s["it"]
        s["ids"][slot] = req.rid
        self.log.append(("join", self.clock.t, req.rid, slot))
        return True

    def finish_slot(self, s, slot):
        assert self.remaining(s, slot) == 0
        self.log.append(("done", self.clock.t, s["ids"][slot]))
        return np.full(3, s["ids"][slot], dtype=np.float32)

    def close(self, s):
        if s in self.open_sessions:
            self.open_sessions.remove(s)
            self.log.append(("close", self.clock.t, tuple(s["ids"])))

    def gradients(self, reqs, model):
        self.cache = self.gradient_bytes
        self.grad_batches.append(tuple(r.rid for r in reqs))
        return [(float(r.rid), np.full(3, r.rid)) for r in reqs]

    def cached_bytes(self):
        return self.cache

    def drop_cache(self):
        if self.cache:
            self.drops += 1
        self.cache = 0


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
    # 4 + 1 on model m (no slot of the first is free when the fifth is admitted), 1 on model other
    assert len(opens) == 3
    assert not [e for e in ex.log if e[0] == "join"]
    assert all(np.all(r.result == r.rid) for r in reqs)
    assert rep.summary()["p99_s"] >= rep.summary()["p50_s"] >= 0
    assert not ex.open_sessions  # every session closed


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
    assert late.admitted < long.done  # admitted while the long session was running
    assert late.done < long.done
    assert late.done - late.arrival < long.done - long.arrival


def test_same_key_arrivals_join_free_slots_of_a_running_session():
    """Four slots: A and B open the session with two idle slots; C and D
    arrive while A and B run and join the idle slots at the next round; E
    arrives after A and B completed, while C and D run, and takes a slot that
    A freed.  One session serves all five, and each slot is advanced exactly
    to its completion."""
    clk = FakeClock()
    ex = FakeExecutor(clk)
    a, b = _req(0), _req(1)
    c, d = _req(2, arrival=0.01), _req(3, arrival=0.02)
    e = _req(4, arrival=0.105)
    srv = serving.Server({"m": None}, executor=ex, chunk=30, max_batch=4)
    rep = srv.run([a, b, c, d, e], clock=clk, sleep=clk.sleep)
    assert len([x for x in ex.log if x[0] == "open"]) == 1
    joins = [x for x in ex.log if x[0] == "join"]
    assert [x[2] for x in joins] == [2, 3, 4]
    assert [x[3] for x in joins] == [2, 3, 0]
    assert c.admitted < a.done and d.admitted < a.done  # joined while A and B ran
    assert e.admitted >= a.done and e.admitted - e.arrival < 0.05
    # a joined shot's service time is its own time axis, not the session's
    assert abs((c.done - c.admitted) - (a.done - a.admitted)) < 0.031
    assert e.done <= rep.makespan
    assert all(np.all(r.result == r.rid) for r in (a, b, c, d, e))


def test_refused_join_opens_a_session_of_its_own():
    """B may not join A's idle slot (the executor refuses, as the C ABI does
    for a source in a taper zone): it opens a session of its own at once."""
    clk = FakeClock()
    ex = FakeExecutor(clk, refuse={1})
    a = _req(0)
    b = _req(1, arrival=0.01)
    srv = serving.Server({"m": None}, executor=ex, chunk=20, max_batch=2)
    srv.run([a, b], clock=clk, sleep=clk.sleep)
    assert all(r.done is not None for r in (a, b))
    assert b.own_session and not a.own_session
    opens = [x for x in ex.log if x[0] == "open"]
    assert len(opens) == 2 and opens[1][2][0] == 1
    assert b.admitted < a.done


def test_gradient_requests_of_one_key_are_evaluated_together():
    clk = FakeClock()
    ex = FakeExecutor(clk)
    g = [_req(i, mode="gradient") for i in range(5)] + [_req(7, mode="gradient", steps=60)]
    srv = serving.Server({"m": None}, executor=ex, chunk=20, max_batch=3)
    srv.run(g, clock=clk, sleep=clk.sleep)
    # one worker: 3 of the first key, then the 2 left of it, then the other key
    assert ex.grad_batches == [(0, 1, 2), (3, 4), (7,)]
    assert all(r.result[0] == float(r.rid) and np.all(r.result[1] == r.rid) for r in g)


def test_kept_gradient_objective_gives_memory_back():
    clk = FakeClock()
    g = _req(0, mode="gradient")
    gb = serving.session_bytes(g.survey, 1, gradient=True)
    ex = FakeExecutor(clk, gradient_bytes=gb)
    m = _req(1, arrival=0.01)
    one = serving.session_bytes(m.survey, 1)
    srv = serving.Server({"m": None}, executor=ex, chunk=20, max_batch=2, budget_bytes=gb + one // 2)
    srv.run([g, m], clock=clk, sleep=clk.sleep)
    assert g.done is not None and m.done is not None
    assert ex.drops >= 1  # the idle objective was released for the modeling session


def test_session_bytes_grow_with_shots_and_gradient():
    sv = synth.elastic_layered(n=24, nsteps=50, taper=4, rec_stride=6, nshots=1)
    assert serving.session_bytes(sv, 2) > serving.session_bytes(sv, 1)
    assert serving.session_bytes(sv, 1, gradient=True) > serving.session_bytes(sv, 1)


class PollingExecutor(FakeExecutor):
    """A session of model "big" reports its steps finished only on every
    third poll; the others at once."""

    def __init__(self, clock):
        super().__init__(clock)
        self.polls = {}
        self.advances = {}
        self.order = []

    def open_batch(self, reqs, model, slots=None):
        s = super().open_batch(reqs, model, slots)
        s["model"] = reqs[0].model_id
        return s

    def advance(self, s, n):
        self.advances[s["model"]] = self.advances.get(s["model"], 0) + 1
        self.order.append(s["model"])
        self.polls[id(s)] = 0
        return super().advance(s, n)

    def ready(self, s):
        self.polls[id(s)] = self.polls.get(id(s), 0) + 1
        return s["model"] != "big" or self.polls[id(s)] >= 3


def test_idle_sessions_advance_while_a_slow_one_runs():
    clk = FakeClock()
    ex = PollingExecutor(clk)
    big = _req(0, model_id="big", steps=300)
    small = _req(1, model_id="small", steps=300)
    srv = serving.Server({"big": None, "small": None}, executor=ex, chunk=20, max_batch=1)
    srv.run([big, small], clock=clk, sleep=clk.sleep)
    assert big.done is not None and small.done is not None
    assert small.done < big.done
    # the small session took its next chunk whenever it was idle, not once per
    # slow round: between two chunks of the big session it ran several
    runs = "".join("b" if m == "big" else "s" for m in ex.order)
    assert "bsss" in runs and ex.advances["small"] == ex.advances["big"]
    assert all(np.all(r.result == r.rid) for r in (big, small))
