"""Host-side logic on CPU: the C-ABI library loads and exports every entry
point of include/fwi3d_gpu.h, parameter defaults match the reference's
struct param, argument validation maps the reference's successCheck aborts to
status codes, and the multi-rank timing reduction works over gloo."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from fwi3d_b200 import _lib, ops, synth
from fwi3d_b200.param import Param

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    with open(os.path.join(ROOT, "include", "fwi3d_gpu.h")) as f:
        src = f.read()
    return sorted(set(re.findall(r"\b(fwi_[A-Za-z_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = header_functions()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib.EXPORTS)
    assert lib.fwi_version().startswith(b"fwi3d_b200")


def test_param_defaults_match_reference_struct():
    c = _lib.CParam()
    _lib.load().fwi_param_default(C.byref(c))
    p = Param()  # field defaults of src/include/param.hpp:8-71
    assert c.courant == pytest.approx(p.courant) and c.dt == p.dt and c.sub == p.sub
    assert c.sinc_half_length == p.sinc_half_length
    assert list(c.bc) == p.bc and list(c.taper) == p.taper
    assert c.free_surface_stiffness == pytest.approx(p.free_surface_stiffness)
    assert c.taper_strength == pytest.approx(p.taper_strength)
    assert (c.vpmin, c.vpmax, c.vsmin, c.vsmax) == pytest.approx((p.vpmin, p.vpmax, p.vsmin, p.vsmax))


def _create(sv, **over):
    lib = _lib.load()
    par = sv.par.copy()
    for k, v in over.items():
        setattr(par, k, v)
    cp = ops.to_cparam(par)
    g = ops.Domain(sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.nmodels).grid()
    w = np.ascontiguousarray(sv.wavelet, np.float32)
    sx = np.ascontiguousarray(np.asarray(par.sxyz[0], np.float32))
    rx = np.ascontiguousarray(np.asarray(par.rxyz[0], np.float32))
    h = C.c_void_p()
    nm = over.pop("_nmodels", sv.nmodels) if "_nmodels" in over else sv.nmodels
    rc = lib.fwi_op_create(C.byref(h), 0, C.byref(g), nm, C.byref(cp), _lib.fptr(w), 1, w.shape[-1], sv.dt_data,
                           _lib.fptr(sx), rx.shape[0], _lib.fptr(rx))
    if rc == 0:
        lib.fwi_op_destroy(h)
    return rc, lib.fwi_last_error().decode()


def test_create_validates_geometry_and_options():
    sv = synth.acoustic_linear(n=16, nsteps=10, rec_stride=4)
    assert _create(sv)[0] == _lib.FWI_OK
    bad = sv.par.copy()
    rc, msg = _create(sv, sxyz=[[5.0, 0.1, 0.1]])
    assert rc == _lib.FWI_ERR_ARG and "outside" in msg
    rc, msg = _create(sv, rxyz=[[[0.05, 0.05, 9.0, 0, 0]]])
    assert rc == _lib.FWI_ERR_ARG and "Receiver 0" in msg
    # acoustic operators ignore the gauge length (analyzeGeometry sets it to 0)
    assert _create(sv, gl=0.01)[0] == _lib.FWI_OK
    # an elastic DAS channel whose fibre leaves the model is rejected
    ev = synth.elastic_layered(n=16, nsteps=10, taper=2, rec_stride=4, nshots=1)
    rc, msg = _create(ev, gl=0.05, rxyz=[[[0.01, 0.06, 0.06, 0.0, 0.0]]])
    assert rc == _lib.FWI_ERR_ARG and "gauge length" in msg
    assert _create(ev, gl=0.02, rxyz=[[[0.06, 0.06, 0.06, 0.3, 1.0]]])[0] == _lib.FWI_OK
    del bad


def test_create_rejects_tiny_grid_and_bad_parameter_count():
    sv = synth.acoustic_linear(n=10, nsteps=10, rec_stride=4)
    rc, msg = _create(sv)
    assert rc == _lib.FWI_ERR_ARG and "12 points" in msg
    sv = synth.acoustic_linear(n=16, nsteps=10, rec_stride=4)
    lib = _lib.load()
    cp = ops.to_cparam(sv.par)
    g = ops.Domain(16, 16, 16, 0.01, 0.01, 0.01, 4).grid()
    w = np.zeros(11, np.float32)
    h = C.c_void_p()
    rc = lib.fwi_op_create(C.byref(h), 0, C.byref(g), 4, C.byref(cp), _lib.fptr(w), 1, 11, 0.001,
                           _lib.fptr(np.zeros(3, np.float32)), 1, _lib.fptr(np.zeros(5, np.float32)))
    assert rc == _lib.FWI_ERR_ARG


def test_operator_shapes_and_dtype_checks():
    sv = synth.elastic_layered(n=16, nsteps=10, rec_stride=4, nshots=2)
    op = ops.from_survey(sv, 1)
    assert op.range_shape == (3, 16, 11)
    assert op.domain_shape == (3, 16, 16, 16)
    with pytest.raises(_lib.FwiError) as e:
        op.apply_forward(False, sv.model.astype(np.float64), np.zeros(op.range_shape, np.float32))
    assert e.value.code == _lib.FWI_ERR_ARG


def test_forward_without_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    sv = synth.acoustic_linear(n=16, nsteps=10, rec_stride=4)
    op = ops.from_survey(sv)
    with pytest.raises(_lib.FwiError) as e:
        op.forward(False, sv.model)
    assert e.value.code == _lib.FWI_ERR_NOGPU


def test_synthetic_surveys_are_seeded():
    a = synth.elastic_layered(n=16, nsteps=5, nshots=1)
    b = synth.elastic_layered(n=16, nsteps=5, nshots=1)
    assert np.array_equal(a.model, b.model) and np.array_equal(a.wavelet, b.wavelet)
    c = synth.elastic_layered(n=16, nsteps=5, nshots=1, seed=9)
    assert not np.array_equal(a.model, c.model)


def _gloo_worker(rank, world, port, q):
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        q.put((rank, bench.max_over_ranks(10.0 * (rank + 1), world)))
    finally:
        dist.destroy_process_group()


def test_timing_is_max_over_ranks_gloo():
    import multiprocessing as mp
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res == [(0, 20.0), (1, 20.0)]


def test_reference_arm_json_line():
    """bench.py --impl reference runs the reference's CPU build on a bounded
    window and prints one JSON line with the contract's keys."""
    import json
    import subprocess
    import sys

    lib = os.path.join(ROOT, "oracle", "_ref", "libfwi3d_ref_fp32.so")
    if not os.path.exists(lib):
        pytest.skip("reference CPU build not present")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "64",
                          "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
