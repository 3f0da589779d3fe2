"""l-BFGS with FP64 vector algebra on the device.

Mirrors the reference's lbfgs (nlsolver.cpp:1292-1360): the pairs
s_k = m_{k+1} - m_k, y_k = g_{k+1} - g_k with rho_k = s_k.y_k, the two-loop
recursion with gamma = rho_{k-1} / |y_{k-1}|^2 and a diagonal H0 of ones.
The reference keeps the pairs and dot products in data_t (FP32 in its FP32
build); here vectors and reductions are FP64 tensors on the GPU.  The line
search is backtracking on the Armijo condition (the reference uses a
regular-Wolfe search, nlsolver.cpp:185-420).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple

import numpy as np


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("l-BFGS runs its vector algebra on a CUDA device")
    return torch


class LBFGS:
    def __init__(self, n: int, m: int = 5, device: str = "cuda:0"):
        self.torch = _torch()
        self.n, self.m, self.device = n, m, device
        self.s: List = []
        self.y: List = []
        self.rho: List[float] = []

    def _vec(self, a) -> "object":
        t = self.torch
        return t.as_tensor(np.ascontiguousarray(a, dtype=np.float64).ravel(), device=self.device)

    def update(self, m1, m0, g1, g0) -> None:
        """updateSY: append the pair of the last step (oldest dropped past m)."""
        s = self._vec(m1) - self._vec(m0)
        y = self._vec(g1) - self._vec(g0)
        rho = float(self.torch.dot(s, y))
        if len(self.s) == self.m:
            self.s.pop(0), self.y.pop(0), self.rho.pop(0)
        self.s.append(s), self.y.append(y), self.rho.append(rho)

    def direction(self, g) -> np.ndarray:
        """computeHg: returns -H g (float64, host)."""
        t = self.torch
        q = self._vec(g)
        k = len(self.s)
        a = [0.0] * k
        gamma = 1.0
        for i in range(k - 1, -1, -1):
            a[i] = float(t.dot(self.s[i], q)) / self.rho[i]
            q = q - a[i] * self.y[i]
        if k:
            gamma = self.rho[k - 1] / float(t.dot(self.y[k - 1], self.y[k - 1]))
        p = gamma * q
        for i in range(k):
            b = float(t.dot(self.y[i], p)) / self.rho[i]
            p = p + (a[i] - b) * self.s[i]
        return (-p).cpu().numpy()


def step(objective: Callable[[np.ndarray], Tuple[float, np.ndarray]], model: np.ndarray, f0: float,
         g0: np.ndarray, solver: LBFGS, nm: int, alpha0: Optional[float] = None, max_tries: int = 8,
         c1: float = 1e-4) -> Tuple[np.ndarray, float, np.ndarray, float]:
    """One l-BFGS iteration: direction, Armijo backtracking, pair update.

    ``objective(model) -> (f, g)`` with g over the first ``nm`` parameters.
    Returns (model, f, g, alpha)."""
    shape = model.shape
    gflat = np.zeros(model.size, dtype=np.float64)
    gflat[: g0.size] = g0.ravel()
    d = solver.direction(gflat)
    d[g0.size:] = 0.0
    slope = float(np.dot(gflat, d))
    if slope >= 0:  # not a descent direction: fall back to steepest descent
        d = -gflat
        slope = float(np.dot(gflat, d))
    if alpha0 is None:
        alpha0 = 0.01 * float(np.abs(model.ravel()[: g0.size]).max()) / max(float(np.abs(d).max()), 1e-30) \
            if not solver.s else 1.0
    alpha = alpha0
    m0 = model.astype(np.float64).ravel()
    for _ in range(max_tries):
        m1 = (m0 + alpha * d).astype(np.float32).reshape(shape)
        f1, g1 = objective(m1)
        if f1 <= f0 + c1 * alpha * slope:
            g1flat = np.zeros_like(gflat)
            g1flat[: g1.size] = g1.ravel()
            solver.update(m1.ravel(), m0, g1flat, gflat)
            return m1, f1, g1, alpha
        alpha *= 0.5
    raise RuntimeError("line search failed to decrease the objective")
