"""fwi_elastic_step_static: the elastic/VTI step that allocates nothing.

The GPU test compares it with the batched modeling entry point
(fwi_batch_*): a survey with a receiver on every grid node records the
displacement field at every time sample (power-of-two spacings make the
recording exact); the static step, fed two recorded samples, must reproduce
the next sample bit for bit, and, fed its own output, the one after (two
calls in a row).  The file is named to be collected last and
passes alone or after the other tests.  The argument checks run on the CPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from fwi3d_b200 import _lib, ops, synth

MAX_POINTS = 1 << 18


def _grid(nx, ny, nz, d=0.008):
    return _lib.Grid(nx, ny, nz, 0.0, 0.0, 0.0, d, d, d)


def _bc(*v):
    return (C.c_int * 6)(*v)


def test_static_step_rejects_oversize_grid():
    lib = _lib.load()
    dummy = C.c_void_p(256)  # never dereferenced: the size check comes first
    g = _grid(65, 64, 64)
    assert 65 * 64 * 64 > MAX_POINTS
    rc = lib.fwi_elastic_step_static(C.byref(g), 3, _bc(1, 1, 1, 1, 1, 1), 1e-4, dummy, dummy, dummy, dummy, None)
    assert rc == _lib.FWI_ERR_ARG
    assert "static scratch limit" in lib.fwi_last_error().decode()


def test_static_step_rejects_absorbing_faces_and_acoustic():
    lib = _lib.load()
    dummy = C.c_void_p(256)
    g = _grid(24, 24, 24)
    rc = lib.fwi_elastic_step_static(C.byref(g), 3, _bc(1, 2, 1, 1, 1, 1), 1e-4, dummy, dummy, dummy, dummy, None)
    assert rc == _lib.FWI_ERR_UNSUPPORTED
    rc = lib.fwi_elastic_step_static(C.byref(g), 2, _bc(1, 1, 1, 1, 1, 1), 1e-4, dummy, dummy, dummy, dummy, None)
    assert rc == _lib.FWI_ERR_ARG
    rc = lib.fwi_elastic_step_static(C.byref(g), 3, _bc(1, 1, 1, 1, 1, 1), 1e-4, None, dummy, dummy, dummy, None)
    assert rc == _lib.FWI_ERR_ARG


def test_static_step_rejects_overlapping_outputs():
    """next may be prev itself but must overlap neither curr, nor the model,
    nor prev in part (the addresses are checked before any device access)."""
    lib = _lib.load()
    g = _grid(24, 24, 24)
    n = 24 ** 3
    base = 1 << 32
    model, prev, curr = base, base + 16 * n * 4, base + 32 * n * 4
    bc = _bc(1, 1, 1, 1, 1, 1)
    cases = {"curr": curr + 4 * n, "the model": model + 4, "prev in part": prev + 4}
    for what, nxt in cases.items():
        rc = lib.fwi_elastic_step_static(C.byref(g), 3, bc, 1e-4, C.c_void_p(model), C.c_void_p(prev),
                                         C.c_void_p(curr), C.c_void_p(nxt), None)
        assert rc == _lib.FWI_ERR_ARG, what
        assert "overlaps " + what in lib.fwi_last_error().decode(), what


def _survey(nmodels, nsteps, cut):
    """Traction-free box (every face bc 1, no taper), one source whose wavelet
    is zero from sample `cut` on, a displacement receiver on every node."""
    # power-of-two spacing and time step: receiver offsets and resampling
    # positions are exact, so the recorded traces are the field values
    d, dt = 2.0 ** -7, 2.0 ** -11
    if nmodels == 3:
        sv = synth.elastic_layered(n=24, nsteps=nsteps, d=d, dt=dt, taper=0, nshots=1)
    else:
        sv = synth.vti_layered(nx=24, ny=26, nz=22, nsteps=nsteps, d=d, dt=dt, taper=0, nshots=1)
    p = sv.par
    p.set_bc(1, 1, 1, 1, 1, 1).set_taper(0, 0, 0, 0, 0, 0)
    p.seismotype = 0
    p.resampling = "linear"
    p.sxyz = [[0.5 * (sv.nx - 1) * sv.dx, 0.4 * (sv.ny - 1) * sv.dy, 0.3 * (sv.nz - 1) * sv.dz]]
    p.rxyz = [[[float(ix * sv.dx), float(iy * sv.dy), float(iz * sv.dz), 0.0, 0.0]
               for iy in range(sv.ny) for ix in range(sv.nx) for iz in range(sv.nz)]]
    w = synth.ricker(40.0, sv.dt_data, nsteps + 1)
    w[cut:] = 0.0
    sv.wavelet = w.astype(np.float32)
    return sv


def _converted(sv):
    """The model as the library converts it (host_ops convert_model), in float32."""
    m = np.asarray(sv.model, dtype=np.float32)
    vp, vs, rho = m[0], m[1], m[2]
    lam = rho * (vp * vp - np.float32(2) * vs * vs)
    mu = rho * vs * vs
    out = [lam, mu, rho]
    if sv.nmodels == 6:
        lpm = lam + mu
        c13 = (np.sqrt((np.float32(2) * (lam + np.float32(2) * mu) * lpm * m[3] + lpm * lpm).astype(np.float64))
               - mu.astype(np.float64)).astype(np.float32)
        c66 = (np.float32(1) + np.float32(2) * m[5]) * mu
        out += [c13, m[4], c66]
    return np.ascontiguousarray(np.stack(out).astype(np.float32))


def _recorded_fields(sv):
    """All time samples of the displacement field, [nt][3][ny][nx][nz], and the propagation dt."""
    lib = _lib.load()
    dom = ops.Domain(sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.nmodels, sv.ox, sv.oy, sv.oz)
    w = np.ascontiguousarray(sv.wavelet, dtype=np.float32)
    sx = np.ascontiguousarray(np.asarray(sv.par.sxyz, dtype=np.float32))
    rx = np.ascontiguousarray(np.asarray(sv.par.rxyz, dtype=np.float32).reshape(1, -1, 5))
    nr = rx.shape[1]
    model = np.ascontiguousarray(sv.model, dtype=np.float32)
    cp = ops.to_cparam(sv.par)
    b = C.c_void_p()
    _lib.check(lib.fwi_batch_create(C.byref(b), 0, C.byref(dom.grid()), sv.nmodels, C.byref(cp), _lib.fptr(model),
                                    _lib.fptr(w), 1, w.shape[-1], sv.dt_data, 1, _lib.fptr(sx), nr, _lib.fptr(rx)))
    try:
        info = _lib.OpInfo()
        lps = C.c_int()
        _lib.check(lib.fwi_batch_get_info(b, C.byref(info), C.byref(lps)))
        assert info.nt == w.shape[-1], "the propagation grid must equal the data sampling for this comparison"
        _lib.check(lib.fwi_batch_reset(b))
        _lib.check(lib.fwi_batch_run(b, info.nt - 1))
        out = np.zeros((1, 3, nr, info.nt), dtype=np.float32)
        _lib.check(lib.fwi_batch_traces(b, _lib.fptr(out)))
    finally:
        lib.fwi_batch_destroy(b)
    f = out[0].reshape(3, sv.ny, sv.nx, sv.nz, info.nt)
    return np.ascontiguousarray(np.moveaxis(f, -1, 0)), float(info.dt)


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.gpu
@pytest.mark.parametrize("nmodels", [3, 6])
def test_static_step_matches_batch_two_calls(nmodels):
    import torch

    nsteps, cut = 90, 60
    sv = _survey(nmodels, nsteps, cut)
    u, dt = _recorded_fields(sv)
    k = 80
    assert np.abs(u[k]).max() > 0
    lib = _lib.load()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    model = torch.from_numpy(_converted(sv)).to(dev)
    prev = torch.from_numpy(u[k - 2]).to(dev)
    curr = torch.from_numpy(u[k - 1]).to(dev)
    out1 = torch.empty_like(curr)
    out2 = torch.empty_like(curr)
    g = _grid(sv.nx, sv.ny, sv.nz, sv.dx)
    bc = _bc(1, 1, 1, 1, 1, 1)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(lib.fwi_elastic_step_static(C.byref(g), nmodels, bc, dt, model.data_ptr(), prev.data_ptr(),
                                           curr.data_ptr(), out1.data_ptr(), stream))
    _lib.check(lib.fwi_elastic_step_static(C.byref(g), nmodels, bc, dt, model.data_ptr(), curr.data_ptr(),
                                           out1.data_ptr(), out2.data_ptr(), stream))
    torch.cuda.synchronize(dev)
    o1, o2 = out1.cpu().numpy(), out2.cpu().numpy()
    # the same per-point kernels on the same inputs: bit-identical
    assert np.array_equal(o1, u[k]) and np.array_equal(o2, u[k + 1]), (_rel(o1, u[k]), _rel(o2, u[k + 1]))
    # a warm call takes no device memory: the free memory of the device and
    # the caching allocator's figures are the same before and after it
    free0, _ = torch.cuda.mem_get_info(dev)
    alloc0 = torch.cuda.memory_allocated(dev)
    _lib.check(lib.fwi_elastic_step_static(C.byref(g), nmodels, bc, dt, model.data_ptr(), out1.data_ptr(),
                                           out2.data_ptr(), prev.data_ptr(), stream))
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0 and torch.cuda.memory_allocated(dev) == alloc0
