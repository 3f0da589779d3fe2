"""Serving loop: continuous batching of modeling and gradient shots.

Requests (one shot each, on a registered model) arrive over time.  A
dispatcher admits them while device memory allows -- each admission is
charged the device bytes of the session it opens, against a budget that
defaults to the device's free memory -- and keeps models and wavefield state
resident until the request completes:

* modeling shots that share a model, a time axis and a receiver count are
  admitted together as one batch session (fwi_batch_*): one kernel launch per
  operator per time step advances all its shots;
* sessions advance `chunk` time steps per scheduling round, each on its own
  CUDA stream, so work of different sessions overlaps on the device and
  requests that arrive meanwhile are admitted at the next round, while the
  others are running;
* gradient shots run the device FWI objective (forward with stored
  snapshots, adjoint, imaging) on worker threads with their own streams.

Latency is completion minus arrival; the report gives p50/p99 beside the
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


class GpuExecutor:
    """Runs sessions through the C ABI on one device."""

    def __init__(self, device: int = 0):
        self.device = device
        self.lib = _lib.load()

    def free_bytes(self) -> int:
        import torch

        free, _ = torch.cuda.mem_get_info(self.device)
        return int(free)

    def open_batch(self, reqs: List[Request], model: np.ndarray):
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
                                             ncomp, w.shape[-1], sv.dt_data, len(reqs), _lib.fptr(sx), nr,
                                             _lib.fptr(rx)))
        _lib.check(self.lib.fwi_batch_reset(h))
        info = _lib.OpInfo()
        _lib.check(self.lib.fwi_batch_get_info(h, C.byref(info), None))
        return {"h": h, "left": info.nt - 1, "nt": info.nt, "nrcomp": info.nrcomp, "nr": nr, "ns": len(reqs),
                "nt_data": w.shape[-1], "points": sv.nx * sv.ny * sv.nz}

    def advance(self, s, nsteps: int) -> int:
        k = min(nsteps, s["left"])
        _lib.check(self.lib.fwi_batch_run(s["h"], k))
        s["left"] -= k
        return k

    def wait(self, s) -> None:
        _lib.check(self.lib.fwi_batch_sync(s["h"]))

    def finish(self, s) -> List[np.ndarray]:
        out = np.zeros((s["ns"], s["nrcomp"], s["nr"], s["nt_data"]), dtype=np.float32)
        _lib.check(self.lib.fwi_batch_traces(s["h"], _lib.fptr(out)))
        self.lib.fwi_batch_destroy(s["h"])
        s["h"] = C.c_void_p()
        return [out[i] for i in range(s["ns"])]

    def gradient(self, req: Request, model: np.ndarray):
        obj = ops.FwiObjective(req.survey, req.observed, normalize=True, batch=1, device=self.device)
        try:
            return obj.evaluate(model)
        finally:
            obj.close()


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
    the reference's (vp, vs, rho[, ...]) parametrisation."""

    def __init__(self, models: Dict[str, np.ndarray], executor=None, budget_bytes: Optional[int] = None,
                 chunk: int = 50, max_batch: int = 8, gradient_workers: int = 1):
        self.models = models
        self.ex = executor if executor is not None else GpuExecutor()
        self.budget = budget_bytes
        self.chunk = chunk
        self.max_batch = max_batch
        self.workers = gradient_workers

    def run(self, requests: List[Request], clock=time.perf_counter, sleep=time.sleep) -> Report:
        budget = self.budget if self.budget is not None else int(self.ex.free_bytes() * 0.9)
        pending: List[Request] = []
        future = sorted(requests, key=lambda r: r.arrival)
        sessions: List[Tuple[dict, List[Request], int]] = []   # (session, requests, bytes)
        grads: List[Tuple[Any, Request, int]] = []
        used = 0
        lock = threading.Lock()
        pool = ThreadPoolExecutor(max_workers=self.workers)
        t0 = clock()
        done = 0
        updates = 0
        try:
            while done < len(requests):
                now = clock() - t0
                while future and future[0].arrival <= now:
                    pending.append(future.pop(0))
                # admission: modeling groups first-come first-served, gradients on free workers
                i = 0
                while i < len(pending):
                    r = pending[i]
                    if r.mode == "gradient":
                        if len(grads) >= self.workers:
                            i += 1
                            continue
                        b = session_bytes(r.survey, 1, gradient=True)
                        if used + b > budget and (sessions or grads):
                            i += 1
                            continue
                        pending.pop(i)
                        r.admitted = clock() - t0
                        fut = pool.submit(self.ex.gradient, r, self.models[r.model_id])
                        grads.append((fut, r, b))
                        with lock:
                            used += b
                        continue
                    group = [q for q in pending if q.mode == "modeling" and q.key() == r.key()][: self.max_batch]
                    b = session_bytes(r.survey, len(group))
                    while used + b > budget and len(group) > 1:
                        group = group[:-1]
                        b = session_bytes(r.survey, len(group))
                    if used + b > budget and (sessions or grads):
                        i += 1
                        continue
                    for q in group:
                        pending.remove(q)
                        q.admitted = clock() - t0
                    s = self.ex.open_batch(group, self.models[r.model_id])
                    sessions.append((s, group, b))
                    used += b
                # advance every session one chunk (asynchronous launches on their own streams)
                for s, grp, _ in sessions:
                    k = self.ex.advance(s, self.chunk)
                    for q in grp:
                        q.updates += k * s["points"]
                for s, _, _ in sessions:
                    self.ex.wait(s)
                # completions
                keep = []
                for s, grp, b in sessions:
                    if s["left"] == 0:
                        for q, tr in zip(grp, self.ex.finish(s)):
                            q.result = tr
                            q.done = clock() - t0
                            q.updates += s["points"]  # the extraction of the last sample
                            updates += q.updates
                            done += 1
                        used -= b
                    else:
                        keep.append((s, grp, b))
                sessions = keep
                gkeep = []
                for fut, r, b in grads:
                    if fut.done():
                        r.result = fut.result()
                        r.done = clock() - t0
                        sv = r.survey
                        r.updates = 2 * sv.nx * sv.ny * sv.nz * (sv.nt_data - 1)
                        updates += r.updates
                        done += 1
                        with lock:
                            used -= b
                    else:
                        gkeep.append((fut, r, b))
                grads = gkeep
                if not sessions and done < len(requests):
                    if grads:
                        sleep(0.002)  # gradients on the workers, nothing to advance here
                    elif future and not pending:
                        sleep(max(0.0, min(0.05, future[0].arrival - (clock() - t0))))
        finally:
            pool.shutdown(wait=True)
        makespan = clock() - t0
        return Report(len(requests), makespan, updates, [r.done - r.arrival for r in requests],
                      [r.done - r.admitted for r in requests], [r.admitted - r.arrival for r in requests])
