"""GPU path against the committed golden fixtures (outputs of the reference's
own CPU build, tests/golden/make_golden.py): traces within 1e-5 relative L2
of the FP32 build, gradients within 1e-4; the distance to the FP64 build is
checked against the reference's own FP32 distance to it."""
import json
import os
import sys

import numpy as np
import pytest

from fwi3d_b200 import ops

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _cases():
    with open(os.path.join(GOLD, "index.json")) as f:
        return sorted(json.load(f))


@pytest.mark.parametrize("name", _cases())
def test_gpu_matches_golden(name):
    import make_golden

    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    sv, grad = make_golden.build(name)
    op = ops.from_survey(sv)
    d = op.forward(False, sv.model)
    e32 = rel(d, g["traces_fp32"])
    e64 = rel(d, g["traces_fp64"])
    ref_gap = rel(g["traces_fp32"], g["traces_fp64"])
    assert e32 < 1e-5, e32
    # no further from the FP64 build than the reference's FP32 build is, up to 2x
    assert e64 < 2 * ref_gap + 1e-6, (e64, ref_gap)
    if grad:
        adj = make_golden.adjoint_data(g["traces_fp32"].shape, float(np.abs(g["traces_fp32"]).max()))
        gr = op.jacobianT(False, None, sv.model, adj)
        for k in range(g["grad_fp32"].shape[0]):
            assert rel(gr[k], g["grad_fp32"][k]) < 1e-4, f"parameter {k}"
        assert rel(gr, g["grad_fp64"]) < 2 * rel(g["grad_fp32"], g["grad_fp64"]) + 1e-5
