#!/usr/bin/env python
"""Benchmark of the wave-propagation hot path on B200 GPUs.

Workload (N=1): elastic isotropic modeling on a 256^3 grid (8 m spacing,
dt 0.6 ms), 8 shots with explosive moment-tensor sources batched on the shared
model, 128x128 three-component velocity receivers, free-surface top and
absorbing sides with 20-point tapers -- seeded synthetic layered model (the
reference publishes no dataset).  One bench step = one time step of the
8-shot batch = 8 * 256^3 grid-point updates.

Our arm: K time steps timed with CUDA events on the engine's stream after W
warm-up steps, run as the library runs them (three-step CUDA graphs
replayed); all state resident in HBM (the working set, ~5 GB, is far larger
than L2, so no flush is needed between steps).  The roofline figure comes
from K further steps with plain launches whose main kernel is timed launch
by launch with events on the same stream.  e2e: the public C-ABI
batch call (fwi_forward_batch) with host buffers on a 300-step time axis,
host<->device copies and host-side preparation inside the timed region
(after one untimed warm-up call of the same kind).

Reference arm (--impl reference): the reference's own CPU code (built from
its sources into oracle/_ref) on the host cores, one shot of the same
workload over a bounded time window.

Multi-GPU (torchrun): shots are independent -- every rank runs its own 8-shot
batch (weak scaling), no collective on the data path; the timing is the max
over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_UPDATE = 48  # algorithmic FP32 traffic of one elastic point update (lambda, mu, rho, prev x3, curr x3, next x3)
# per physics: algorithmic bytes per update (acoustic: K, 1/rho, prev, curr read, next written; VTI: six
# model arrays + nine wavefield values) and the modeling configuration of the benchmark
PHYSICS = {
    "elastic": {"bytes": 48, "shots": 8, "n": 256},
    "acoustic": {"bytes": 20, "shots": 1, "n": 101},
    "vti": {"bytes": 60, "shots": 24, "n": 0},  # 320 x 320 x 200 (n > 0: a cube of n for profiling)
}


_CACHE = {}


def workload(n=256, nshots=8, nsteps=3000, physics="elastic"):
    """The seeded survey; the model is generated once per grid size and the
    wavelet cut to ``nsteps`` + 1 samples."""
    from fwi3d_b200 import synth

    key = (physics, n)
    if key not in _CACHE:
        if physics == "elastic":
            _CACHE[key] = synth.elastic_layered(n=n, nsteps=4000, nshots=8)
        elif physics == "acoustic":
            _CACHE[key] = synth.acoustic_linear(n=n, nsteps=4000)
        else:
            dims = dict(nx=n, ny=n, nz=n) if n > 0 else {}
            _CACHE[key] = synth.vti_layered(nsteps=4000, nshots=24, **dims)
    base = _CACHE[key]
    sv = base.shot(0) if nshots == 1 else base
    sv = synth.Survey(sv.name, sv.nmodels, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.model,
                      np.ascontiguousarray(base.wavelet[:nsteps + 1]), sv.dt_data, sv.par.copy())
    if nshots != 1:
        sv.par.sxyz = sv.par.sxyz[:nshots]
        sv.par.rxyz = sv.par.rxyz[:nshots]
        sv.par.ns = nshots
    return sv


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_update(physics):
    """DRAM bytes per grid-point update of the step's main kernels for one
    physics, from the committed ncu summary (profiles/ncu_traffic.txt:
    `<physics>.<key>=value` lines): (bytes per update, kernel name)."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        vals = {}
        with open(path) as f:
            for line in f:
                if "=" in line and not line.startswith("#"):
                    k, v = line.strip().split("=", 1)
                    vals[k.strip()] = v.strip()
        return float(vals[f"{physics}.dram_bytes_per_update"]), vals.get(f"{physics}.kernel", "")
    except Exception:
        return None, ""


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"fwi3d_b200_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 7:
                    continue
                try:
                    sm.append(float(parts[0]))
                    smax = float(parts[1])
                except ValueError:
                    continue
                for name, v in zip(names, parts[3:7]):
                    if v.lower() == "active":
                        reasons.add(name)
        try:
            os.remove(self.path)
        except OSError:
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(value, world, device=None):
    """Max of a per-rank scalar over all ranks (the timing rule for N > 1);
    works with the nccl (device tensor) and gloo (CPU tensor) backends."""
    if world <= 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def cpu_reference(n_steps, threads, n=256, physics="elastic", short=10):
    """Reference CPU code (oracle/_ref, built from the reference sources): one
    shot of the workload, timed over a `short`-step and an `n_steps`-step
    window of the unmodified apply_forward; the difference is the time of
    n_steps - short steps of its propagate() loop, so model analysis and
    set-up (timed separately) are not in the rate.  Returns (pt-updates/s,
    seconds per step, set-up seconds)."""
    from oracle import refpy

    def timed(k):
        sv = workload(n=n, nshots=1, nsteps=k, physics=physics)
        t0 = time.perf_counter()
        refpy.modeling(sv, shot=0, precision="fp32", nthreads=threads)
        return sv.nxyz, time.perf_counter() - t0

    n_steps = max(n_steps, short + 4)
    _, t1 = timed(short)
    nxyz, t2 = timed(n_steps)
    per_step = max(t2 - t1, 1e-9) / (n_steps - short)
    return nxyz / per_step, per_step, max(0.0, t1 - short * per_step)


def grid_label(sv):
    return f"{sv.nx}^3" if sv.nx == sv.ny == sv.nz else f"{sv.nx}x{sv.ny}x{sv.nz}"


def workload_label(physics, sv, ns, nr):
    g = grid_label(sv)
    d = sv.dx * 1000
    if physics == "elastic":
        return (f"elastic iso modeling {g}, {d:g} m, dt {sv.dt_data * 1e3:g} ms, {ns} moment-tensor shots batched on "
                f"the shared model, {nr} 3-C receivers per shot")
    if physics == "acoustic":
        return (f"acoustic VD modeling {g}, {d:g} m, dt {sv.dt_data * 1e3:g} ms, {ns} shot, {nr} pressure receivers, "
                f"20-point tapers, free-surface top")
    return (f"elastic VTI modeling {g}, {d:g} m, dt {sv.dt_data * 1e3:g} ms, {ns} vertical-force shots batched on "
            f"the shared model, {nr} 3-C receivers per shot")


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    k = max(20, min(args.steps, args.ref_cap))  # the reference needs nt >= 10 (we_op.cpp:621, 838)
    if args.warmup > 0:
        cpu_reference(14, threads, n=args.n, physics=args.physics, short=10)
    value, per_step, setup = cpu_reference(k, threads, n=args.n, physics=args.physics)
    sv = workload(n=args.n, nshots=1, nsteps=k, physics=args.physics)
    sample = (f"1 shot of the {grid_label(sv)} {args.physics} workload: the unmodified apply_forward timed over a "
              f"10-step and a {k}-step window, rate from the difference ({k - 10} steps of propagate(); set-up "
              f"{setup:.2f} s excluded), OMP threads={threads}")
    line = {
        "impl": "reference", "metric": "grid-pt updates/s", "value": value, "unit": "pt/s", "n_gpus": args.gpus,
        "steps": k - 10, "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_label(args.physics, sv, PHYSICS[args.physics]["shots"], len(sv.par.rxyz[0]))
                   + " (CPU: 1-shot bounded window)",
                   "grid": [sv.nx, sv.ny, sv.nz], "shots": PHYSICS[args.physics]["shots"], "parallelism": "cpu"},
        "cpu_baseline": {"value": value, "unit": "pt/s", "cores": threads, "kind": "reference", "sample": sample,
                         "setup_s": setup},
        "e2e": {"value": value, "unit": "pt/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local):
    import ctypes as C

    import torch

    from fwi3d_b200 import _lib, ops

    torch.cuda.set_device(local)
    lib = _lib.load()
    sv = workload(n=args.n, nshots=args.shots, nsteps=max(2 * args.steps + args.warmup + 1, 301), physics=args.physics)
    ns = len(sv.par.sxyz)
    dom = ops.Domain(sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.nmodels)
    bpu = PHYSICS[args.physics]["bytes"]
    nrcomp = 1 if sv.nmodels == 2 else 3
    nr = len(sv.par.rxyz[0])
    w = np.ascontiguousarray(sv.wavelet, dtype=np.float32)
    sx = np.ascontiguousarray(np.asarray(sv.par.sxyz, dtype=np.float32))
    rx = np.ascontiguousarray(np.asarray(sv.par.rxyz, dtype=np.float32))
    model = np.ascontiguousarray(sv.model, dtype=np.float32)
    cp = ops.to_cparam(sv.par)

    h = C.c_void_p()
    _lib.check(lib.fwi_batch_create(C.byref(h), local, C.byref(dom.grid()), sv.nmodels, C.byref(cp), _lib.fptr(model),
                                    _lib.fptr(w), 1, w.shape[-1], sv.dt_data, ns, _lib.fptr(sx), nr, _lib.fptr(rx)))
    sp = C.c_void_p()
    _lib.check(lib.fwi_batch_stream(h, C.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value)
    info = _lib.OpInfo()
    lps = C.c_int()
    _lib.check(lib.fwi_batch_get_info(h, C.byref(info), C.byref(lps)))
    _lib.check(lib.fwi_batch_reset(h))
    _lib.check(lib.fwi_batch_run(h, args.warmup))
    _lib.check(lib.fwi_batch_sync(h))
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    # timed region 1 (value): K steps as a user runs them (CUDA-graph replay)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    _lib.check(lib.fwi_batch_run(h, args.steps))
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    # timed region 2 (roofline): K more steps with the step's main kernel timed
    # launch by launch with events on the engine stream (plain launches)
    _lib.check(lib.fwi_batch_time_main_kernel(h, args.steps))
    _lib.check(lib.fwi_batch_run(h, args.steps))
    k_ms, k_n, k_pts, k_name = C.c_double(), C.c_int(), C.c_int64(), C.c_char_p()
    _lib.check(lib.fwi_batch_main_kernel_time(h, C.byref(k_ms), C.byref(k_n), C.byref(k_pts), C.byref(k_name)))
    _lib.check(lib.fwi_batch_time_main_kernel(h, 0))
    clk = clocks.stop()
    if world > 1:
        ms = max_over_ranks(ms, world, device="cuda")
        torch.distributed.barrier()
    lib.fwi_batch_destroy(h)

    units_per_step = ns * sv.nxyz  # per rank
    value = world * units_per_step * args.steps / (ms / 1e3)
    ms_step = ms / args.steps
    peak, peak_kind = peaks()
    launch_ms = k_ms.value / max(1, k_n.value)
    kernel = (k_name.value or b"").decode()
    achieved = bpu * k_pts.value / (launch_ms * 1e-3) / 1e9 if k_n.value else None
    step_gbs = bpu * units_per_step / (ms_step / 1e3) / 1e9
    tpu, tkernel = traffic_per_update(args.physics)

    # e2e through the public C-ABI call, host buffers, 300-step time axis
    e2e = None
    if not args.no_e2e:
        sv_e = workload(n=args.n, nshots=args.shots, nsteps=300, physics=args.physics)
        we = np.ascontiguousarray(sv_e.wavelet, dtype=np.float32)
        out = np.zeros((ns, nrcomp, nr, we.shape[-1]), dtype=np.float32)

        def e2e_call():
            _lib.check(lib.fwi_forward_batch(local, C.byref(dom.grid()), sv.nmodels, C.byref(cp), _lib.fptr(model),
                                             _lib.fptr(we), 1, we.shape[-1], sv_e.dt_data, ns, _lib.fptr(sx), nr,
                                             _lib.fptr(rx), _lib.fptr(out)))

        e2e_call()  # untimed warm-up call (first-use costs of the path's kernels and host tables)
        if world > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        e2e_call()
        te = time.perf_counter() - t0
        te = max_over_ranks(te, world, device="cuda")
        nsteps_e = we.shape[-1] - 1
        h2d = model.nbytes + we.nbytes + sx.nbytes + rx.nbytes
        e2e = {"value": world * units_per_step * nsteps_e / te, "unit": "pt/s",
               "h2d_bytes_per_step": h2d / nsteps_e, "d2h_bytes_per_step": out.nbytes / nsteps_e,
               "steps": nsteps_e, "seconds": te, "warmup_calls": 1}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        v, per_step, setup = cpu_reference(args.cpu_steps, threads, n=args.n, physics=args.physics)
        cpu = {"value": v, "unit": "pt/s", "cores": threads, "kind": "reference", "setup_s": setup,
               "sample": f"reference CPU build, 1 shot of the {grid_label(sv)} {args.physics} workload, "
                         f"apply_forward over 10- and {max(args.cpu_steps, 14)}-step windows, rate from the "
                         f"difference ({per_step:.3f} s per step; set-up {setup:.2f} s excluded), "
                         f"OMP threads={threads}"}

    if rank == 0:
        line = {
            "metric": "grid-pt updates/s", "value": value, "unit": "pt/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered model, Ricker sources)",
            "config": {"workload": workload_label(args.physics, sv, ns, nr),
                       "grid": [sv.nx, sv.ny, sv.nz], "shots_per_gpu": ns, "receivers_per_shot": nr,
                       "parallelism": f"shots x{world} (weak)", "l2": "working set >> L2 (no flush needed)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak if achieved else None), "peak_kind": peak_kind,
                         "traffic": (tpu * k_pts.value if tpu and tkernel == kernel else None),
                         "kernel": kernel, "launch_ms": launch_ms, "launches": k_n.value,
                         "updates_per_launch": k_pts.value,
                         "algorithmic_bytes_per_update": bpu,
                         "step_achieved_gbs": step_gbs,
                         "note": f"achieved = {bpu} B x updates per launch / mean CUDA-event time of the main kernel's "
                                 "launches in a second timed region of K steps run with plain launches (the first, "
                                 "which gives value, replays CUDA graphs); traffic = ncu DRAM bytes per update of that kernel "
                                 "(profiles/ncu_traffic.txt) x updates per launch; step_achieved_gbs covers every "
                                 "kernel of the step"},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(lps.value) * args.steps, "clocks": clk,
        }
        # the configuration's other two measures, run after the timed modeling
        # region: FWI gradients/hour and the serving mix's p50/p99
        if world == 1 and not args.no_gradient:
            line["gradient"] = gradient_block(args.n_grad, args.steps_grad, args.shots_side, args.grad_batch or 4,
                                              device=local)
        if world == 1 and not args.no_serving:
            line["serving"] = serving_block(args.requests, args.rate, device=local)
        print(json.dumps(line), flush=True)
    return 0


def gradient_survey(n, nsteps, nside):
    """Elastic FWI problem of the gradient workload: layered background with
    three +-8 % Gaussian anomalies (true model), smoothed initial model,
    nside x nside shots, 2-point receiver stride, seeded."""
    from fwi3d_b200 import synth

    sv = synth.elastic_anomaly(n=n, nsteps=nsteps, nshots_side=nside, rec_stride=2)
    sv.par.sub = -1
    return sv


def gradient_block(n, nsteps, nside, batch, slots_plain=40, free_frac=0.8, device=0):
    """FWI gradients/hour on the elastic FWI configuration (n^3, 10 m, dt 1 ms,
    nsteps steps, nside^2 shots, 100x100-class receivers).  Full storage of the
    forward wavefield does not fit (FP32: 96 MB per state per shot at 200^3),
    so both forms checkpoint with FP32 restart states (exact recomputation):
      plain: the per-shot operator (forward + jacobianT, one shot per call, as
             a caller of the reference's operator API runs it) with
             `slots_plain` checkpoint slots;
      batched: the device objective with `batch` shots advancing in lockstep
             and as many checkpoint slots as fit `free_frac` of free HBM,
             residual, adjoint sources and FP64 sums on the device.
    Both are timed on the first `batch` shots; shots are independent and of
    equal cost, so gradients/hour scale by nside^2 / batch.  The gradient of
    the batched form is compared with the sum of the plain per-shot ones
    (normalised the same way)."""
    import torch

    from fwi3d_b200 import ops, synth

    sv = gradient_survey(n, nsteps, nside)
    ns_all = len(sv.par.sxyz)
    sv.par.sxyz = sv.par.sxyz[:batch]
    sv.par.rxyz = sv.par.rxyz[:batch]
    sv.par.ns = batch
    true = synth.Survey(sv.name, 3, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.extra["true_model"], sv.wavelet,
                        sv.dt_data, sv.par.copy())
    obs = ops.forward_batch(true, device=device)
    model = np.ascontiguousarray(sv.model, dtype=np.float32)
    dt = sv.dt_data
    dnorm = float(np.sum(obs.astype(np.float64) ** 2)) * dt

    def ht(r):
        a = (r * np.float32(dt)).astype(np.float32)
        a[..., 0] = (r[..., 0].astype(np.float64) * 0.5 * dt).astype(np.float32)
        a[..., -1] = (r[..., -1].astype(np.float64) * 0.5 * dt).astype(np.float32)
        return a

    # plain: per-shot operators, FP32 checkpoints
    sp = sv.par.copy()
    sp.checkpoint_slots = slots_plain
    svp = synth.Survey(sv.name, 3, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, model, sv.wavelet, dt, sp)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    g_plain = np.zeros((3,) + model.shape[1:], dtype=np.float64)
    for s in range(batch):
        op = ops.from_survey(svp, s, device=device)
        r = op.forward(False, model) - obs[s]
        g_plain += op.jacobianT(False, None, model, ht(r))
        op.close()
    t_plain = time.perf_counter() - t0
    g_plain /= dnorm

    # batched: device objective, checkpoint slots sized to the free memory
    free, _ = torch.cuda.mem_get_info(device)
    sv.par.snapshot_budget_gb = free_frac * free / 1e9
    obj = ops.FwiObjective(sv, obs, batch=batch, device=device)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    f_b, g_b = obj.evaluate(model)
    t_b = time.perf_counter() - t0
    dev_bytes = obj.device_bytes()
    obj.close()
    diff = float(np.linalg.norm(g_b - g_plain) / max(np.linalg.norm(g_plain), 1e-30))
    scale = ns_all / batch
    return {
        "metric": "FWI gradients/hour", "value": 3600.0 / (t_b * scale), "unit": "gradients/h",
        "workload": f"elastic FWI gradient {n}^3, 10 m, dt 1 ms, {nsteps} steps, {ns_all} shots "
                    f"({nside}x{nside}), 2-point receiver stride, sub 1; timed on {batch} shots, scaled by "
                    f"{ns_all}/{batch}",
        "form": f"device objective, {batch} shots per launch, FP32 restart checkpoints (binomial schedule) in "
                f"{free_frac:.0%} of free HBM, FP64 misfit and gradient sums",
        "seconds_per_batch": t_b, "device_bytes": dev_bytes,
        "plain": {"value": 3600.0 / (t_plain * scale), "unit": "gradients/h", "seconds_per_batch": t_plain,
                  "form": f"per-shot operator (forward + jacobianT), FP32 restart checkpoints, {slots_plain} slots"},
        "speedup_vs_plain": t_plain / t_b,
        "gradient_rel_l2_vs_plain": diff,
        "misfit": f_b,
    }


def vti_gradient_block(nsample=2, nsteps=3000, precision=2, slots_plain=40, free_frac=0.8, device=0):
    """FWI gradients/hour on the VTI configuration (320 x 320 x 200, 10 m,
    dt 0.8 ms, nsteps steps, 24 shots, 160 x 160 receivers): the device
    objective with `nsample` shots per launch and per-(state, level, shot,
    component) scaled 16-bit restart checkpoints (precision 2 FP16, 1 BF16)
    in `free_frac` of free HBM, against the per-shot operator with
    `slots_plain` FP32 checkpoint slots.  Timed on `nsample` shots and scaled
    by 24 / nsample (shots are independent and of equal cost).  Observed data:
    the model with a 3 % faster top half.  The 16-bit checkpoints' gradient
    error against the FP64 reference is the reduced-size oracle case of
    tests/test_gpu_checkpoint.py."""
    import torch

    from fwi3d_b200 import ops, synth

    sv = synth.vti_layered(nsteps=nsteps)
    ns_all = len(sv.par.sxyz)
    sv.par.sxyz = sv.par.sxyz[:nsample]
    sv.par.rxyz = sv.par.rxyz[:nsample]
    sv.par.ns = nsample
    sv.par.sub = -1
    true_m = sv.model.copy()
    true_m[0, :, :, : sv.nz // 2] *= np.float32(1.03)
    true = synth.Survey(sv.name, 6, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, true_m, sv.wavelet, sv.dt_data,
                        sv.par.copy())
    obs = ops.forward_batch(true, device=device)
    model = np.ascontiguousarray(sv.model, dtype=np.float32)
    dt = sv.dt_data
    dnorm = float(np.sum(obs.astype(np.float64) ** 2)) * dt

    def ht(r):
        a = (r * np.float32(dt)).astype(np.float32)
        a[..., 0] = (r[..., 0].astype(np.float64) * 0.5 * dt).astype(np.float32)
        a[..., -1] = (r[..., -1].astype(np.float64) * 0.5 * dt).astype(np.float32)
        return a

    sp = sv.par.copy()
    sp.checkpoint_slots = slots_plain
    svp = synth.Survey(sv.name, 6, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, model, sv.wavelet, dt, sp)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    g_plain = None
    for s in range(nsample):
        op = ops.from_survey(svp, s, device=device)
        r = op.forward(False, model) - obs[s]
        g = op.jacobianT(False, None, model, ht(r)).astype(np.float64)
        g_plain = g if g_plain is None else g_plain + g
        op.close()
    t_plain = time.perf_counter() - t0
    g_plain /= dnorm

    free, _ = torch.cuda.mem_get_info(device)
    sv.par.snapshot_budget_gb = free_frac * free / 1e9
    sv.par.checkpoint_precision = precision
    obj = ops.FwiObjective(sv, obs, batch=nsample, device=device)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    f_b, g_b = obj.evaluate(model)
    t_b = time.perf_counter() - t0
    dev_bytes = obj.device_bytes()
    obj.close()
    diff = float(np.linalg.norm(g_b - g_plain) / max(np.linalg.norm(g_plain), 1e-30))
    scale = ns_all / nsample
    pname = {1: "BF16", 2: "FP16"}[precision]
    return {
        "metric": "FWI gradients/hour", "value": 3600.0 / (t_b * scale), "unit": "gradients/h",
        "workload": f"elastic VTI FWI gradient {sv.nx}x{sv.ny}x{sv.nz}, 10 m, dt 0.8 ms, {nsteps} steps, "
                    f"{ns_all} shots, {len(sv.par.rxyz[0])} receivers per shot; timed on {nsample} shots, scaled "
                    f"by {ns_all}/{nsample}",
        "form": f"device objective, {nsample} shots per launch, scaled {pname} restart checkpoints (binomial "
                f"schedule) in {free_frac:.0%} of free HBM, FP64 misfit and gradient sums",
        "seconds_per_batch": t_b, "device_bytes": dev_bytes,
        "plain": {"value": 3600.0 / (t_plain * scale), "unit": "gradients/h", "seconds_per_batch": t_plain,
                  "form": f"per-shot operator (forward + jacobianT), FP32 restart checkpoints, {slots_plain} slots"},
        "speedup_vs_plain": t_plain / t_b,
        "gradient_rel_l2_vs_plain_fp32": diff,
        "misfit": f_b,
    }


def serving_block(nreq, rate, device=0):
    """Serving mix shaped like the serving configuration, scaled to a bounded
    run: Poisson arrivals, six models of the three physics at uneven grids,
    modeling and gradient shots; throughput and p50/p99 latency (service and
    queueing reported apart)."""
    from fwi3d_b200 import servemix, serving

    models, reqs = servemix.make_mix(nreq=nreq, rate=rate, seed=5, grids=servemix.BENCH_GRIDS,
                                     steps=servemix.BENCH_STEPS, rec=servemix.BENCH_REC, p_gradient=0.25)
    srv = serving.Server(models, chunk=100, max_batch=8, gradient_workers=2)
    rep = srv.run(reqs)
    s = rep.summary()
    return {
        "metric": "serving grid-pt updates/s", "value": s["gpt_per_s"] * 1e9, "unit": "pt/s",
        "workload": f"{nreq} requests (of the configuration's 512), Poisson {rate}/s, acoustic/elastic/VTI x 2 models, "
                    f"grids {servemix.BENCH_GRIDS}, steps {servemix.BENCH_STEPS}, 8-15 Hz, receiver lines "
                    f"{servemix.BENCH_REC}, 25 % gradients (FP32 checkpoints)",
        "requests_per_s": s["requests_per_s"], "p50_s": s["p50_s"], "p99_s": s["p99_s"],
        "service_p50_s": s["service_p50_s"], "service_p99_s": s["service_p99_s"],
        "queue_p50_s": s["queue_p50_s"], "queue_p99_s": s["queue_p99_s"], "makespan_s": s["seconds"],
        "latency_unit": "s",
    }


def run_gradient(args):
    if args.physics == "vti":
        line = vti_gradient_block(args.grad_batch or 2, args.steps_grad_vti)
        dtype, data = "f32 stencils, scaled FP16 checkpoints, FP64 sums", "synthetic (seeded layered VTI model)"
    else:
        line = gradient_block(args.n_grad, args.steps_grad, args.shots_side, args.grad_batch or 4)
        dtype, data = "f32 stencils, FP32 checkpoints, FP64 sums", "synthetic (seeded layered model + 3 anomalies)"
    line.update({"n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": line["seconds_per_batch"] * 1e3,
                 "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                 "dtype": dtype, "data": data, "config": {"workload": line["workload"]}})
    print(json.dumps(line), flush=True)
    return 0


def run_serving(args):
    line = serving_block(args.requests, args.rate)
    line.update({"n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": line["makespan_s"] * 1e3,
                 "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                 "data": "synthetic (seeded request mix)", "config": {"workload": line["workload"]}})
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=30)
    ap.add_argument("--ref-cap", type=int, default=40, help="max time steps of the CPU reference window")
    ap.add_argument("--physics", default="elastic", choices=sorted(PHYSICS),
                    help="modeling workload: elastic 256^3 x 8 shots (default), acoustic 101^3 x 1, "
                         "vti 320x320x200 x 24")
    ap.add_argument("--n", type=int, default=None, help="grid points per axis (profiling runs use smaller grids)")
    ap.add_argument("--shots", type=int, default=None)
    ap.add_argument("--workload", default="modeling", choices=["modeling", "gradient", "serving"])
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--n-grad", type=int, default=200)
    ap.add_argument("--steps-grad", type=int, default=2500)
    ap.add_argument("--no-gradient", action="store_true", help="skip the gradients/hour block of the default line")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving block of the default line")
    ap.add_argument("--shots-side", type=int, default=4)
    ap.add_argument("--grad-batch", type=int, default=None,
                    help="shots per launch of the gradient workload (elastic 4, VTI 2)")
    ap.add_argument("--steps-grad-vti", type=int, default=3000)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.n is None:
        args.n = PHYSICS[args.physics]["n"]
    if args.shots is None:
        args.shots = PHYSICS[args.physics]["shots"]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "gradient":
        return run_gradient(args)
    if args.workload == "serving":
        return run_serving(args)
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        return run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
