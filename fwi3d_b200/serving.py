"""Serving loop: continuous batching of modeling and gradient shots.

Requests (one shot each, on a registered model) arrive over time.  A
dispatcher admits them while device memory allows -- each admission is
charged the device bytes of the session it opens, against a budget that
defaults to the device's free memory -- and keeps models and wavefield state
resident until the request completes:

* modeling shots that share a model, a time axis and a receiver count are
  admitted together as one batch session (fwi_batch_*): one kernel launch per
  operator per time step advances all its shots;
* a session's shots are slots with their own start steps: a shot that
  arrives while a session of its key runs takes a free slot (a spare one, or
  one whose shot has completed) at the next scheduling round and starts
  there, while the other slots run on; idle slots cost memory, not compute;
* a session gets up to `chunk` time steps at a time (to its next slot
  completion) on its own CUDA stream, and its next steps as soon as those
  have finished: the dispatcher polls the sessions instead of waiting for
  all of them, so a small session is not held to the pace of a large one,
  work of different sessions overlaps on the device, and requests that
  arrive meanwhile are admitted while the others run;
* gradient requests of one key (same model, time axis, receiver count) are
  evaluated together, one objective per shot from the same batched launches
  (fwi_objective_evaluate_shots), on worker threads with their own streams;
  an objective is kept per key and batch size after its requests, so the
  next gradients of that key reuse its device buffers (no cudaMalloc /
  cudaFree, which would synchronise the device under the running sessions),
  and it gives its memory back when an admission needs it.

Latency is completion minus arrival; the report gives p50/p99 of it, of the
service time (completion minus admission) and of the queueing time beside the
throughput.  The scheduler talks to an executor object, so its admission and
batching logic is testable without a GPU.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional, Tuple

import numpy as np

from . import _lib, ops


@dataclass
class Request:
    rid: int
    model_id: str
    mode: str                      # "modeling" or "gradient"
    survey: Any                    # synth.Survey of one shot (model taken from the registry)
    observed: Optional[np.ndarray] = None   # gradient: [1][nrcomp][nr][nt_data]
    arrival: float = 0.0           # seconds after the start of the run
    admitted: Optional[float] = None
    done: Optional[float] = None
    result: Any = None
    updates: int = 0               # grid-point updates performed for it
    own_session: bool = False      # refused by a running session's slot (opens its own)

    def key(self) -> Tuple:
        """Shots with equal keys can share a batch session: same model, time
        axis, receiver count, wavelet and propagation parameters."""
        sv = self.survey
        p = sv.par
        w = np.ascontiguousarray(sv.wavelet, dtype=np.float32)
        return (self.model_id, sv.nt_data, float(sv.dt_data), len(p.rxyz[0]), sv.nmodels, hash(w.tobytes()),
                tuple(p.bc), tuple(p.taper), bool(p.mt), p.seismotype, p.resampling, float(p.courant), float(p.dt),
                float(p.fangle), float(p.fazimuth), (p.mxx, p.myy, p.mzz, p.mxy, p.mxz, p.myz))


def session_bytes(sv, nshots: int, gradient: bool = False) -> int:
    """Device bytes a batch session (or a gradient evaluation) of `nshots`
    shots holds: wavefields, derivative scratch, model, traces, and for a
    gradient the FP16 snapshot residuals, their FP64 codec state and the
    decode ring; 10 % margin for tables."""
    n = sv.nx * sv.ny * sv.nz
    nc = 1 if sv.nmodels == 2 else 3
    nt = sv.nt_data  # propagation samples are at least this many
    nr = len(sv.par.rxyz[0])
    b = 3 * nshots * nc * n * 4 + sv.nmodels * n * 4 + nc * nshots * nr * nt * 4
    if sv.nmodels != 2:
        b += nshots * 9 * n * 4
    if gradient:
        slots = int(getattr(sv.par, "checkpoint_slots", 0))
        if slots > 0:
            # FP32 restart states (two levels), recomputation levels, ring, zero snapshot
            b += (2 * slots + 7) * nshots * nc * n * 4 + 3 * n * 8
        else:
            nsnap = nt + 1
            b += nsnap * nshots * nc * n * 2 + 2 * nshots * nc * n * 8 + 4 * nshots * nc * n * 4 + 3 * n * 8
    return int(b * 1.1)


def combined_survey(reqs: List[Request]):
    """One survey of the requests' shots (same key): their sources and
    receiver lines in request order, and their observed data stacked."""
    from . import synth

    sv = reqs[0].survey
    par = sv.par.copy()
    par.sxyz = [list(r.survey.par.sxyz[0]) for r in reqs]
    par.rxyz = [list(r.survey.par.rxyz[0]) for r in reqs]
    par.ns = len(reqs)
    comb = synth.Survey(sv.name, sv.nmodels, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.model, sv.wavelet,
                        sv.dt_data, par)
    obs = None
    if all(r.observed is not None for r in reqs):
        obs = np.concatenate([np.asarray(r.observed, dtype=np.float32).reshape((1,) + np.shape(r.observed)[-3:])
                              for r in reqs])
    return comb, obs


class GpuExecutor:
    """Runs sessions through the C ABI on one device.  A session's shots are
    slots (fwi_batch_enable_slots / fwi_batch_join / fwi_batch_release): a
    free slot takes a new shot of the same key at the session's current step
    while the other slots run on.  Gradient objectives are kept per request
    key and batch size between requests (fwi_objective_set_shots), so that
    gradients of a key seen before allocate nothing on the device."""

    def __init__(self, device: int = 0, max_cached: int = 1):
        self.device = device
        self.lib = _lib.load()
        self.max_cached = max_cached
        self._gcache: Dict[Tuple, Tuple[Any, int]] = {}   # (key, batch) -> (objective, bytes), least recent first
        self._glock = threading.Lock()

    def free_bytes(self) -> int:
        import torch

        free, _ = torch.cuda.mem_get_info(self.device)
        return int(free)

    @staticmethod
    def _geometry(req: Request):
        p = req.survey.par
        sx = np.ascontiguousarray(np.asarray(p.sxyz[0][:3], dtype=np.float32))
        rx = np.ascontiguousarray(np.asarray(p.rxyz[0], dtype=np.float32))
        return sx, rx

    def open_batch(self, reqs: List[Request], model: np.ndarray, slots: Optional[int] = None):
        """A session of `slots` (>= len(reqs)) shot slots, the first len(reqs)
        running the requests from step 0, the others idle until a shot joins."""
        nreal = len(reqs)
        slots = max(nreal, slots or nreal)
        reqs = list(reqs) + [reqs[0]] * (slots - nreal)  # geometry of the idle slots: never run
        sv = reqs[0].survey
        dom = ops.Domain(sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.nmodels, sv.ox, sv.oy, sv.oz)
        w = np.ascontiguousarray(sv.wavelet, dtype=np.float32)
        ncomp = 1 if w.ndim == 1 else w.shape[0]
        sx = np.ascontiguousarray(np.asarray([r.survey.par.sxyz[0][:3] for r in reqs], dtype=np.float32))
        rx = np.ascontiguousarray(np.asarray([r.survey.par.rxyz[0] for r in reqs], dtype=np.float32))
        nr = rx.shape[1]
        cp = ops.to_cparam(sv.par)
        h = C.c_void_p()
        _lib.check(self.lib.fwi_batch_create(C.byref(h), self.device, C.byref(dom.grid()), sv.nmodels, C.byref(cp),
                                             _lib.fptr(np.ascontiguousarray(model, dtype=np.float32)), _lib.fptr(w),
                                             ncomp, w.shape[-1], sv.dt_data, slots, _lib.fptr(sx), nr, _lib.fptr(rx)))
        try:
            _lib.check(self.lib.fwi_batch_reset(h))
            _lib.check(self.lib.fwi_batch_enable_slots(h))
            for k in range(nreal, slots):
                _lib.check(self.lib.fwi_batch_release(h, k))
            info = _lib.OpInfo()
            _lib.check(self.lib.fwi_batch_get_info(h, C.byref(info), None))
        except Exception:
            self.lib.fwi_batch_destroy(h)
            raise
        return {"h": h, "nt": info.nt, "nrcomp": info.nrcomp, "nr": nr, "ns": slots, "nt_data": w.shape[-1],
                "points": sv.nx * sv.ny * sv.nz}

    def advance(self, s, nsteps: int) -> int:
        _lib.check(self.lib.fwi_batch_run(s["h"], nsteps))
        return nsteps

    def wait(self, s) -> None:
        _lib.check(self.lib.fwi_batch_sync(s["h"]))

    def ready(self, s) -> bool:
        """The session's enqueued steps have finished (without waiting)."""
        r = C.c_int()
        _lib.check(self.lib.fwi_batch_ready(s["h"], C.byref(r)))
        return bool(r.value)

    def remaining(self, s, slot: int) -> int:
        left = C.c_int()
        _lib.check(self.lib.fwi_batch_slot_time(s["h"], slot, None, C.byref(left)))
        return left.value

    def join(self, s, slot: int, req: Request) -> bool:
        sx, rx = self._geometry(req)
        rc = self.lib.fwi_batch_join(s["h"], slot, _lib.fptr(sx), _lib.fptr(rx))
        if rc == _lib.FWI_ERR_UNSUPPORTED:
            return False  # a source in a taper zone: it opens a session of its own
        _lib.check(rc)
        return True

    def finish_slot(self, s, slot: int) -> np.ndarray:
        """Data of the slot's completed shot; the slot turns idle."""
        out = np.zeros((s["nrcomp"], s["nr"], s["nt_data"]), dtype=np.float32)
        _lib.check(self.lib.fwi_batch_slot_traces(s["h"], slot, _lib.fptr(out)))
        _lib.check(self.lib.fwi_batch_release(s["h"], slot))
        return out

    def close(self, s) -> None:
        if s["h"]:
            self.lib.fwi_batch_destroy(s["h"])
            s["h"] = C.c_void_p()

    def cached_bytes(self) -> int:
        """Device bytes held by the gradient objectives kept between requests."""
        with self._glock:
            return sum(b for _, b in self._gcache.values())

    def drop_cache(self) -> None:
        with self._glock:
            items = list(self._gcache.values())
            self._gcache.clear()
        for obj, _ in items:
            obj.close()

    def gradients(self, reqs: List[Request], model: np.ndarray) -> List[Tuple[float, np.ndarray]]:
        """(misfit, gradient) of each request (same key), one objective per
        shot from one batched evaluation; the objective is kept afterwards."""
        sv, obs = combined_survey(reqs)
        key = (reqs[0].model_id,) + reqs[0].key() + (int(getattr(sv.par, "checkpoint_slots", 0)), len(reqs))
        with self._glock:
            hit = self._gcache.pop(key, None)
        obj = hit[0] if hit else None
        try:
            if obj is None:
                obj = ops.FwiObjective(sv, obs, normalize=True, batch=len(reqs), device=self.device)
            else:
                obj.set_shots(sv, obs)
            f, g = obj.evaluate_shots(model)
        except Exception:
            if obj is not None:
                obj.close()
            raise
        evict = []
        with self._glock:
            self._gcache[key] = (obj, session_bytes(sv, len(reqs), gradient=True))
            while len(self._gcache) > self.max_cached:
                evict.append(self._gcache.pop(next(iter(self._gcache)))[0])
        for o in evict:
            o.close()
        return [(float(f[k]), g[k]) for k in range(len(reqs))]


@dataclass
class Report:
    requests: int
    makespan: float
    updates: int
    latencies: List[float] = field(default_factory=list)   # completion - arrival
    service: List[float] = field(default_factory=list)     # completion - admission
    queueing: List[float] = field(default_factory=list)    # admission - arrival

    def summary(self) -> Dict[str, float]:
        def pct(v, q):
            a = np.asarray(v, dtype=np.float64)
            return float(np.percentile(a, q)) if a.size else 0.0

        return {"requests": self.requests, "seconds": self.makespan,
                "gpt_per_s": self.updates / self.makespan / 1e9 if self.makespan > 0 else 0.0,
                "requests_per_s": self.requests / self.makespan if self.makespan > 0 else 0.0,
                "p50_s": pct(self.latencies, 50), "p99_s": pct(self.latencies, 99),
                "service_p50_s": pct(self.service, 50), "service_p99_s": pct(self.service, 99),
                "queue_p50_s": pct(self.queueing, 50), "queue_p99_s": pct(self.queueing, 99)}


class Server:
    """Dispatcher of one device.  `models` maps model ids to host arrays in
    the reference's (vp, vs, rho[, ...]) parametrisation.  `max_batch`
    bounds the shots of a modeling session and of a gradient evaluation;
    `slots` (default max_batch) is the number of shot slots a modeling
    session opens with, so that later shots of its key can join it."""

    def __init__(self, models: Dict[str, np.ndarray], executor=None, budget_bytes: Optional[int] = None,
                 chunk: int = 50, max_batch: int = 8, gradient_workers: int = 1, slots: Optional[int] = None):
        self.models = models
        self.ex = executor if executor is not None else GpuExecutor()
        self.budget = budget_bytes
        self.chunk = chunk
        self.max_batch = max_batch
        self.workers = gradient_workers
        self.slots = max_batch if slots is None else max(1, min(slots, max_batch))

    def run(self, requests: List[Request], clock=time.perf_counter, sleep=time.sleep) -> Report:
        budget = self.budget if self.budget is not None else int(self.ex.free_bytes() * 0.9)
        pending: List[Request] = []
        future = sorted(requests, key=lambda r: r.arrival)
        sessions: List[Dict[str, Any]] = []   # {"x": executor session, "key", "slots": [Request|None], "bytes"}
        grads: List[Tuple[Any, List[Request], int]] = []
        used = 0
        lock = threading.Lock()
        pool = ThreadPoolExecutor(max_workers=self.workers)
        cached = getattr(self.ex, "cached_bytes", lambda: 0)
        t0 = clock()
        done = 0
        updates = 0

        def fits(b: int) -> bool:
            # device memory of a new session or gradient evaluation; the idle
            # gradient objectives kept between requests give their memory back
            # when it is needed; with nothing running, anything is admitted
            if used + cached() + b <= budget:
                return True
            if cached():
                self.ex.drop_cache()
            return used + b <= budget or not (sessions or grads)

        def arrivals():
            now = clock() - t0
            while future and future[0].arrival <= now:
                pending.append(future.pop(0))

        try:
            while done < len(requests):
                arrivals()
                # admission: gradients of one key together on a free worker;
                # modeling shots join a free slot of a running session of their
                # key, else open a session with the pending shots of that key
                # (first come, first served)
                i = 0
                while i < len(pending):
                    r = pending[i]
                    key = r.key()
                    if r.mode == "gradient":
                        if len(grads) >= self.workers:
                            i += 1
                            continue
                        group = [q for q in pending if q.mode == "gradient" and q.key() == key][: self.max_batch]
                        b = session_bytes(r.survey, len(group), gradient=True)
                        while used + b > budget and len(group) > 1:
                            group = group[:-1]
                            b = session_bytes(r.survey, len(group), gradient=True)
                        if not fits(b):
                            i += 1
                            continue
                        for q in group:
                            pending.remove(q)
                            q.admitted = clock() - t0
                        fut = pool.submit(self.ex.gradients, group, self.models[r.model_id])
                        grads.append((fut, group, b))
                        with lock:
                            used += b
                        continue
                    joined = False
                    if not r.own_session:
                        for se in sessions:
                            if se["key"] != key or se.get("busy"):
                                continue
                            for k, q in enumerate(se["slots"]):
                                if q is None:
                                    if self.ex.join(se["x"], k, r):
                                        se["slots"][k] = r
                                        joined = True
                                    else:
                                        r.own_session = True
                                    break
                            if joined or r.own_session:
                                break
                    if joined:
                        pending.pop(i)
                        r.admitted = clock() - t0
                        continue
                    group = [q for q in pending if q.mode == "modeling" and q.key() == key][: self.max_batch]
                    cap = max(len(group), self.slots)
                    b = session_bytes(r.survey, cap)
                    while used + cached() + b > budget and cap > len(group):
                        cap -= 1
                        b = session_bytes(r.survey, cap)
                    while used + b > budget and len(group) > 1:
                        group = group[:-1]
                        cap = len(group)
                        b = session_bytes(r.survey, cap)
                    if not fits(b):
                        i += 1
                        continue
                    for q in group:
                        pending.remove(q)
                        q.admitted = clock() - t0
                    x = self.ex.open_batch(group, self.models[r.model_id], cap)
                    sessions.append({"x": x, "key": key, "slots": list(group) + [None] * (cap - len(group)),
                                     "bytes": b})
                    used += b
                # every idle session gets its steps to its next slot completion,
                # at most one chunk (asynchronous launches on its own stream)
                for se in sessions:
                    if se.get("busy"):
                        continue
                    act = [k for k, q in enumerate(se["slots"]) if q is not None]
                    if not act:
                        continue  # kept for a pending shot of its key, which joins next round
                    k = min([self.chunk] + [self.ex.remaining(se["x"], j) for j in act])
                    if k > 0:
                        self.ex.advance(se["x"], k)
                        se["busy"] = True
                    for j in act:
                        se["slots"][j].updates += k * se["x"]["points"]
                # poll: sessions whose steps have finished turn idle
                ready = getattr(self.ex, "ready", None)
                progressed = False
                for se in sessions:
                    if se.get("busy") and (ready is None or ready(se["x"])):
                        if ready is None:
                            self.ex.wait(se["x"])
                        se["busy"] = False
                        progressed = True
                # completions of the idle sessions; a session without shots
                # closes unless a pending shot of its key will take a slot at
                # the next admission
                arrivals()
                keep = []
                for se in sessions:
                    if se.get("busy"):
                        keep.append(se)
                        continue
                    for j, q in enumerate(se["slots"]):
                        if q is not None and self.ex.remaining(se["x"], j) == 0:
                            q.result = self.ex.finish_slot(se["x"], j)
                            q.done = clock() - t0
                            updates += q.updates
                            done += 1
                            se["slots"][j] = None
                    waiting = any(q.mode == "modeling" and q.key() == se["key"] and not q.own_session for q in pending)
                    if all(q is None for q in se["slots"]) and not waiting:
                        self.ex.close(se["x"])
                        used -= se["bytes"]
                    else:
                        keep.append(se)
                sessions = keep
                gkeep = []
                for fut, group, b in grads:
                    if fut.done():
                        res = fut.result()
                        for r, out in zip(group, res):
                            r.result = out
                            r.done = clock() - t0
                            sv = r.survey
                            r.updates = 2 * sv.nx * sv.ny * sv.nz * (sv.nt_data - 1)
                            updates += r.updates
                            done += 1
                        with lock:
                            used -= b
                    else:
                        gkeep.append((fut, group, b))
                grads = gkeep
                if sessions and not progressed and all(se.get("busy") for se in sessions):
                    sleep(0.0005)  # every session's steps still running
                elif not sessions and done < len(requests):
                    if grads:
                        sleep(0.002)  # gradients on the workers, nothing to advance here
                    elif future and not pending:
                        sleep(max(0.0, min(0.05, future[0].arrival - (clock() - t0))))
        finally:
            pool.shutdown(wait=True)
            for se in sessions:
                if se.get("busy"):
                    self.ex.wait(se["x"])
                self.ex.close(se["x"])
            if hasattr(self.ex, "drop_cache"):
                self.ex.drop_cache()
        makespan = clock() - t0
        return Report(len(requests), makespan, updates, [r.done - r.arrival for r in requests],
                      [r.done - r.admitted for r in requests], [r.admitted - r.arrival for r in requests])
