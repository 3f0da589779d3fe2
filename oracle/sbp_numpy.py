"""Dense-matrix restatement of the 4th-order SBP operators (numpy).

TEST INFRASTRUCTURE ONLY: used by tests/ to check the summation-by-parts
identities of the coefficient tables the GPU kernels are built from.

Restated from the operator definitions of nmbader/fwi3d:
  D1 with its 4-row closure      src/cpp/spatial_operators.cpp:179-210
  D2var with its 6-row closure   src/include/spatial_operators.hpp:34-96
  H quadrature                   src/cpp/spatial_operators.cpp:11-53
  boundary derivative S          src/include/spatial_operators.hpp:241
The closure weights are read from the product's table source
(fwi3d_b200/csrc/sbp_d2_closure.inc) so the test checks the very numbers the
kernels use.
"""
from __future__ import annotations

import os
import re
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
INC = os.path.join(os.path.dirname(HERE), "fwi3d_b200", "csrc", "sbp_d2_closure.inc")

D1B = [[Fraction(-24, 17), Fraction(59, 34), Fraction(-4, 17), Fraction(-3, 34), 0, 0],
       [Fraction(-1, 2), 0, Fraction(1, 2), 0, 0, 0],
       [Fraction(4, 43), Fraction(-59, 86), 0, Fraction(59, 86), Fraction(-4, 43), 0],
       [Fraction(3, 98), 0, Fraction(-59, 98), 0, Fraction(32, 49), Fraction(-4, 49)]]
HQ = [Fraction(17, 48), Fraction(59, 48), Fraction(43, 48), Fraction(49, 48)]
D2IN = [Fraction(-3, 4), Fraction(-5, 6), Fraction(-1, 24), Fraction(1, 6), Fraction(1, 2),
        Fraction(1, 2), Fraction(1, 6), Fraction(-1, 8), Fraction(1, 6), Fraction(-1, 8)]


def d2_closure():
    """[6][8][8] closure weights (row, field sample, material sample) from the .inc file."""
    b = np.zeros((6, 8, 8))
    pat = re.compile(r"D2B\((\d+), (\d+), (\d+), (-?\d+), (\d+)\)")
    with open(INC) as f:
        for m in pat.finditer(f.read()):
            r, j, k, p, q = map(int, m.groups())
            b[r, j, k] = p / q
    return b


def h_matrix(n, h=1.0):
    d = np.ones(n)
    for i in range(4):
        d[i] = d[n - 1 - i] = float(HQ[i])
    return np.diag(d * h)


def d1_matrix(n, h=1.0):
    D = np.zeros((n, n))
    for i in range(n):
        if i < 4:
            D[i, :6] = [float(x) for x in D1B[i]]
        elif i >= n - 4:
            D[i, n - 6:] = [-float(x) for x in D1B[n - 1 - i]][::-1]
        else:
            D[i, i - 2:i + 3] = [1 / 12, -2 / 3, 0, 2 / 3, -1 / 12]
    return D / h


def d2var_matrix(f, h=1.0):
    """Matrix of the variable-coefficient second derivative for coefficient samples f."""
    n = len(f)
    B = d2_closure()
    c = [float(x) for x in D2IN]
    D = np.zeros((n, n))
    for i in range(n):
        if i < 6 or i >= n - 6:
            hi = i >= n - 6
            r = n - 1 - i if hi else i
            for j in range(8):
                v = sum(B[r, j, k] * f[n - 1 - k if hi else k] for k in range(8))
                D[i, n - 1 - j if hi else j] += v
        else:
            fm2, fm1, f0, fp1, fp2 = f[i - 2:i + 3]
            D[i, i] = c[0] * f0 + c[1] * (fm1 + fp1) + c[2] * (fm2 + fp2)
            D[i, i - 1] = c[3] * fm2 + c[4] * fm1 + c[5] * f0 + c[6] * fp1
            D[i, i + 1] = c[3] * fp2 + c[4] * fp1 + c[5] * f0 + c[6] * fm1
            D[i, i - 2] = c[7] * fm2 + c[8] * fm1 + c[9] * f0
            D[i, i + 2] = c[7] * fp2 + c[8] * fp1 + c[9] * f0
    return D / (h * h)
