"""The CPU oracle: the reference's own library (oracle/_ref) pinned against the
golden fixtures made from it, and the SBP identities of the coefficient tables."""
import json
import os

import numpy as np
import pytest

from oracle import sbp_numpy

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_oracle_libraries_precisions(oracle_fp32):
    assert oracle_fp32._lib("fp32").oracle_data_t_size() == 4
    if oracle_fp32.available("fp64"):
        assert oracle_fp32._lib("fp64").oracle_data_t_size() == 8


def _golden_cases():
    with open(os.path.join(GOLD, "index.json")) as f:
        return sorted(json.load(f))


@pytest.mark.parametrize("name", _golden_cases())
def test_oracle_reproduces_golden(oracle_fp32, name):
    import sys
    sys.path.insert(0, GOLD)
    import make_golden

    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    sv, grad = make_golden.build(name)
    d32, info = oracle_fp32.modeling(sv, precision="fp32")
    assert rel(d32, g["traces_fp32"]) < 1e-6
    # the reference's own FP32 error, stated by the FP64 build
    assert rel(g["traces_fp32"], g["traces_fp64"]) < 1e-4
    if grad:
        adj = make_golden.adjoint_data(d32.shape, float(np.abs(d32).max()))
        _, g32, _ = oracle_fp32.forward_jacobianT(sv, adj, precision="fp32")
        assert rel(g32, g["grad_fp32"]) < 1e-6
        assert rel(g["grad_fp32"], g["grad_fp64"]) < 1e-3


@pytest.mark.parametrize("n", [12, 16, 29])
def test_sbp_d1_summation_by_parts(n):
    """H D1 + (H D1)^T = diag(-1, 0, ..., 0, 1): the SBP property of the D1 closure."""
    H, D = sbp_numpy.h_matrix(n), sbp_numpy.d1_matrix(n)
    Q = H @ D
    B = np.zeros((n, n))
    B[0, 0], B[-1, -1] = -1, 1
    assert np.abs(Q + Q.T - B).max() < 1e-12


@pytest.mark.parametrize("n", [13, 20, 33])
def test_sbp_d2var_symmetric_and_exact(n):
    """Variable-coefficient SBP property of the D2 closure: with d0, dn the
    boundary derivative rows (3rd-order one-sided, the SAT's S up to sign),
    H D2(b) + b0 e0 d0^T - bn en dn^T is symmetric (it is -M(b)); D2 annihilates
    constants and is exact on quadratics in the interior."""
    rng = np.random.default_rng(n)
    f = 1.0 + 0.3 * rng.random(n)
    H = sbp_numpy.h_matrix(n)
    D2 = sbp_numpy.d2var_matrix(f)
    s = np.array([11 / 6, -3, 1.5, -1 / 3])
    d0 = np.zeros(n)
    d0[:4] = -s
    dn = np.zeros(n)
    dn[-4:] = s[::-1]
    M = H @ D2 + f[0] * np.outer(np.eye(n)[0], d0) - f[-1] * np.outer(np.eye(n)[-1], dn)
    assert np.abs(M - M.T).max() < 1e-9
    assert np.abs(D2 @ np.ones(n)).max() < 1e-10
    x = np.arange(n, dtype=float)
    D2c = sbp_numpy.d2var_matrix(np.ones(n))
    assert np.abs((D2c @ (x * x))[6:-6] - 2).max() < 1e-9
