"""Non-linear solvers of the FWI loop: l-BFGS, NLCG and steepest descent with
the reference's line searches, vector algebra in FP64 on the device.

Mirrors nmbader/fwi3d src/cpp/nlsolver.cpp and src/include/nlsolver.hpp:

* ``quadratic`` / ``cubic`` step interpolation (nlsolver.cpp:10-35);
* ``WeakWolfe`` -- sufficient decrease with quadratic then cubic backtracking
  (nlsolver.cpp:37-182), the solvers' default line search;
* ``RegularWolfe`` -- sufficient decrease and curvature condition with the
  bracketing phase and ``zoom`` (nlsolver.cpp:185-420), the default of the
  reference's FWI program (``lsearch=regular_wolfe``, param.hpp:55);
* ``Lbfgs`` -- updateSY / computeHg two-loop recursion with gamma =
  rho_{m-1}/|y_{m-1}|^2 and a diagonal H0 (nlsolver.cpp:1158-1360);
* ``Nlcg`` -- Fletcher-Reeves, Polak-Ribiere, PR+ (nlsolver.cpp:815-945);
* ``Nlsd`` -- steepest descent.

Each iteration's control flow, stopping rules, trial counting and step-length
formulas are the reference's.  The reference keeps vectors and dot products in
its data_t (FP32 in its FP32 build); here every vector and reduction is FP64
(torch on the GPU by default), and the model is handed to the objective in
FP32 as the reference's model vector is.

The problem object (``Problem``) plays the reference's ``optimization``
(optimization.hpp): ``res()`` evaluates the objective at the current model,
``get_func()`` returns it and ``grad()`` makes the gradient current.  As in
``nlls_fwi``, one evaluation gives both the misfit and the gradient.
"""
from __future__ import annotations

import math
from typing import Callable, List, Optional, Tuple

import numpy as np

ZERO = 1e-10   # nlsolver.cpp:6
STOL = 1e-3    # nlsolver.cpp:7


class Backend:
    """FP64 vectors: torch tensors on a CUDA device (default), or numpy on the
    host (host-side logic tests without a GPU)."""

    def __init__(self, device: Optional[str] = "cuda:0"):
        self.device = device
        if device is not None:
            import torch

            if not torch.cuda.is_available():
                raise RuntimeError("the solver's vector algebra runs on a CUDA device (device=None: host numpy)")
            self.torch = torch

    def vec(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        if self.device is None:
            return a.copy()
        return self.torch.as_tensor(a, device=self.device)

    def host(self, v) -> np.ndarray:
        return v.copy() if self.device is None else v.cpu().numpy()

    def dot(self, a, b) -> float:
        return float(np.dot(a, b)) if self.device is None else float(self.torch.dot(a, b))

    def norm(self, a) -> float:
        return math.sqrt(self.dot(a, a))

    def copy(self, a):
        return a.copy() if self.device is None else a.clone()


def quadratic(f: float, df: float, stp0: float, f0: float) -> float:
    """Minimiser of the quadratic through (0, f) with slope df and (stp0, f0)
    (nlsolver.cpp:10-16)."""
    if f0 <= f + df * stp0:
        ans = stp0 * 1.1
    else:
        ans = -df * stp0 * stp0 / (2 * (f0 - f - df * stp0))
    if ans / stp0 < STOL or abs(ans - stp0) / stp0 < STOL:
        ans = stp0 / 2.0
    return ans


def cubic(f: float, df: float, stp0: float, f0: float, stp1: float, f1: float) -> float:
    """Minimiser of the cubic through (0, f, df), (stp0, f0), (stp1, f1), with
    the reference's fall-backs (nlsolver.cpp:18-35)."""
    x1 = f1 - f - df * stp1
    x2 = f0 - f - df * stp0
    x3 = stp0 * stp0 * stp1 * stp1 * (stp1 - stp0)
    a = (stp0 * stp0 * x1 - stp1 * stp1 * x2) / x3
    b = (-stp0 * stp0 * stp0 * x1 + stp1 * stp1 * stp1 * x2) / x3
    delta = b * b - 3 * a * df
    step, func = (stp1, f1) if f1 < f0 else (stp0, f0)
    if abs(a) < ZERO or delta < 0:
        ans = quadratic(f, df, step, func)
    else:
        ans = (-b + math.sqrt(delta)) / (3 * a)
    if ans / step < STOL or abs(step - ans) / step < STOL:
        ans = step / 2.0
    elif abs(stp0 + stp1 - step - ans) / (stp0 + stp1 - step) < STOL:
        ans = (stp0 + stp1 - step) / 2.0
    return ans


class Problem:
    """The optimisation problem: model m (FP64 vector), objective
    ``evaluate(model_float32) -> (f, g)`` with g over the first ``ng`` values
    of the model (the propagator's gradient parameters), zero elsewhere."""

    def __init__(self, m0: np.ndarray, evaluate: Callable, backend: Backend):
        self.be = backend
        self.shape = m0.shape
        self.m = backend.vec(m0)
        self.g = backend.vec(np.zeros(m0.size))
        self.evaluate = evaluate
        self.f = None
        self._pending_g = None
        self.nevals = 0

    def model_f32(self) -> np.ndarray:
        return self.be.host(self.m).astype(np.float32).reshape(self.shape)

    def res(self) -> None:
        f, g = self.evaluate(self.model_f32())
        self.nevals += 1
        self.f = float(f)
        gg = np.zeros(int(np.prod(self.shape)), dtype=np.float64)
        gr = np.asarray(g, dtype=np.float64).ravel()
        gg[: gr.size] = gr
        self._pending_g = gg

    def get_func(self) -> float:
        return self.f

    def grad(self) -> None:
        self.g = self.be.vec(self._pending_g)


class WeakWolfe:
    """Sufficient-decrease line search (nlsolver.hpp:28-81, nlsolver.cpp:37-182)."""

    flag_g = True  # the gradient is evaluated after the line search

    def __init__(self, c1: float = 1e-4, a0: float = 1.0, a1: float = 0.0, version: bool = False):
        if not 0 < c1 < 1:
            raise ValueError("The constant c1 must be in (0,1).")
        self.c1, self.a0, self.a1, self.version = c1, a0, a1, version
        self.reset()

    def reset(self):
        self.stp0 = self.stp1 = self.stp = 0.0
        self.f = self.df = self.f0 = self.f1 = 0.0

    def search(self, prob: Problem, m0, p, it: int, max_trial: int, counts: dict, gnorm: float) -> Tuple[bool, float]:
        be = prob.be
        trial = 0
        alpha = 0.0
        while True:
            if trial > max_trial:
                return False, gnorm
            if trial == 0:
                df0 = self.df
                self.f = prob.get_func()
                self.df = be.dot(prob.g, p)
                if it == 0:
                    self.stp0 = self.a0 / gnorm
                    if self.a1 > 0:
                        self.stp0 = max(self.stp0, self.a1 * be.norm(prob.m) / gnorm)
                else:
                    self.stp0 = self.stp * df0 / self.df
                    if self.version:
                        self.stp0 = min(1.0, 1.00001 * (2 * (self.f - self.f0) / self.df))
                trial += 1
                alpha = self.stp0
                continue
            prob.m = m0 + alpha * p
            prob.res()
            counts["feval"] += 1
            f = prob.get_func()
            if f != f:
                raise RuntimeError("the objective function is NaN")
            if trial == 1:
                self.f0 = f
                if f <= self.f + self.c1 * self.stp0 * self.df or f <= ZERO:
                    self.stp, self.f0, self.f = self.stp0, self.f, f
                    return f > ZERO, gnorm
                self.stp1 = quadratic(self.f, self.df, self.stp0, self.f0)
            else:
                if trial > 2:
                    self.f0 = self.f1
                self.f1 = f
                if f <= self.f + self.c1 * self.stp1 * self.df or f <= ZERO:
                    self.f0, self.f, self.stp = self.f, f, self.stp1
                    return f > ZERO, gnorm
                temp = cubic(self.f, self.df, self.stp0, self.f0, self.stp1, self.f1)
                self.stp0, self.stp1 = self.stp1, temp
            alpha = self.stp1
            trial += 1


class RegularWolfe:
    """Line search satisfying the sufficient-decrease and curvature conditions
    (nlsolver.hpp:84-154, nlsolver.cpp:185-420): bracketing phase, then zoom
    with quadratic / cubic interpolation."""

    flag_g = False  # the gradient of the accepted step is already current

    def __init__(self, c1: float = 1e-4, c2: float = 0.9, a0: float = 1.0, a1: float = 0.0,
                 step_max: float = 1e6, version: bool = False):
        if not (0 < c1 < 1 and c1 < c2 < 1):
            raise ValueError("The constants c1, c2 must satisfy 0<c1<c2<1")
        self.c1, self.c2, self.a0, self.a1, self.step_max, self.version = c1, c2, a0, a1, step_max, version
        self.reset()

    def reset(self):
        self.stp0 = self.stp1 = self.stp = 0.0
        self.f = self.df = self.f0 = self.f1 = 0.0

    def _phi(self, prob, m0, p, alpha, counts):
        prob.m = m0 + alpha * p
        prob.res()
        counts["feval"] += 1
        f = prob.get_func()
        if f != f:
            raise RuntimeError("the objective function is NaN")
        return f

    def _dphi(self, prob, p, counts):
        prob.grad()
        counts["geval"] += 1
        return prob.be.norm(prob.g), prob.be.dot(prob.g, p)

    def search(self, prob: Problem, m0, p, it: int, max_trial: int, counts: dict, gnorm: float) -> Tuple[bool, float]:
        be = prob.be
        trial = 0
        df0 = self.df
        self.f = prob.get_func()
        self.df = be.dot(prob.g, p)
        self.stp0 = 0.0
        if it == 0:
            self.f0 = self.f
            self.stp1 = self.a0 / gnorm
            if self.a1 > 0:
                self.stp1 = max(self.stp1, self.a1 * be.norm(prob.m) / gnorm)
        else:
            self.stp1 = self.stp * df0 / self.df
            if self.version:
                self.stp1 = min(1.0, 1.00001 * (2 * (self.f - self.f0) / self.df))
        alpha = self.stp1
        while True:
            if trial >= max_trial:
                return False, gnorm
            f = self._phi(prob, m0, p, alpha, counts)
            trial += 1
            self.f1 = f
            if f <= ZERO:
                self.stp, self.f0, self.f = alpha, self.f, f
                return False, gnorm
            if self.f1 > self.f + self.c1 * alpha * self.df or (self.f1 >= self.f0 and trial > 1):
                return self._zoom(False, prob, m0, p, trial, max_trial, counts, gnorm)
            gnorm, df1 = self._dphi(prob, p, counts)
            if df1 >= self.c2 * self.df:
                self.stp, self.f0, self.f = alpha, self.f, f
                return True, gnorm
            if df1 >= 0:
                return self._zoom(True, prob, m0, p, trial, max_trial, counts, gnorm)
            self.stp0 = self.stp1
            self.stp1 = min(quadratic(self.f, self.df, self.stp1, self.f1), self.step_max)
            alpha = self.stp1
            self.f0 = self.f1

    def _zoom(self, reverse, prob, m0, p, trial, max_trial, counts, gnorm) -> Tuple[bool, float]:
        alo, ahi, flo, fhi = self.stp0, self.stp1, self.f0, self.f1
        if reverse:
            alo, ahi, flo, fhi = self.stp1, self.stp0, self.f1, self.f0
        while True:
            if trial >= max_trial:
                return False, gnorm
            if alo == 0:
                alpha = quadratic(self.f, self.df, ahi, fhi)
            elif ahi == 0:
                alpha = quadratic(self.f, self.df, alo, flo)
            else:
                alpha = cubic(self.f, self.df, alo, flo, ahi, fhi)
            f = self._phi(prob, m0, p, alpha, counts)
            trial += 1
            self.f0, self.f1 = self.f1, f
            if f <= ZERO:
                self.stp, self.f0, self.f = alpha, self.f, f
                return False, gnorm
            if self.f1 > self.f + self.c1 * alpha * self.df or self.f1 >= flo:
                ahi, fhi = alpha, self.f1
            else:
                gnorm, df1 = self._dphi(prob, p, counts)
                if df1 >= self.c2 * self.df:
                    self.stp, self.f0, self.f = alpha, self.f, f
                    return True, gnorm
                if df1 * (ahi - alo) >= 0:
                    ahi, fhi = alo, flo
                alo, flo = alpha, self.f1


class _Solver:
    """Common loop state (nlsolver.hpp:182-230): iterations, trials, threshold,
    function history, evaluation counts."""

    def __init__(self, niter: int, max_trial: int = 10, threshold: float = 0.0, ls=None):
        self.niter, self.max_trial, self.threshold = niter, max_trial, threshold
        self.ls = ls if ls is not None else WeakWolfe(1e-4, 1, 0, False)
        self.func: List[float] = []
        self.counts = {"feval": 0, "geval": 0}
        self.steps: List[float] = []

    def reset(self):
        self.func = []
        self.counts = {"feval": 0, "geval": 0}
        self.steps = []
        self.ls.reset()

    def _start(self, prob: Problem) -> bool:
        self.reset()
        prob.res()
        self.counts["feval"] += 1
        f = prob.get_func()
        self.func.append(f)
        return not (f <= ZERO or f != f)


class Lbfgs(_Solver):
    """l-BFGS (nlsolver.cpp:1158-1360)."""

    def __init__(self, niter: int, max_trial: int = 10, threshold: float = 0.0, ls=None,
                 h0: Optional[np.ndarray] = None, m: int = 5):
        super().__init__(niter, max_trial, threshold, ls)
        if h0 is not None and np.min(h0) <= 0:
            raise ValueError("Initial diagonal inverse Hessian must be definite positive.")
        self.h0, self.m = h0, m

    def run(self, prob: Problem) -> Problem:
        be = prob.be
        if not self._start(prob):
            return prob
        h0 = be.vec(np.ones(prob.m.shape[0]) if self.h0 is None else self.h0)
        s: List = []
        y: List = []
        rho: List[float] = []
        m0 = be.copy(prob.m)
        g0 = None
        k, rate, gnorm, f = 0, 1.0, 999.0, self.func[0]
        success = True
        while k < self.niter and rate > self.threshold and gnorm > ZERO and f > ZERO and success:
            if self.ls.flag_g or k == 0:
                prob.grad()
                self.counts["geval"] += 1
                gnorm = be.norm(prob.g)
            # updateSY: the pair of the last step, the oldest dropped past m
            if k > 0:
                sk, yk = prob.m - m0, prob.g - g0
                if len(s) == self.m:
                    s.pop(0), y.pop(0), rho.pop(0)
                s.append(sk), y.append(yk), rho.append(be.dot(sk, yk))
            # computeHg
            q = be.copy(prob.g)
            a = [0.0] * len(s)
            gamma = 1.0
            for i in range(len(s) - 1, -1, -1):
                a[i] = be.dot(s[i], q) / rho[i]
                q = q - a[i] * y[i]
            if s:
                gamma = rho[-1] / be.dot(y[-1], y[-1])
            p = gamma * h0 * q
            for i in range(len(s)):
                b = be.dot(y[i], p) / rho[i]
                p = p + (a[i] - b) * s[i]
            p = -p
            if be.dot(p, prob.g) >= 0:
                break  # not a descent direction: the solver stops
            if k > 0:
                m0 = be.copy(prob.m)
            g0 = be.copy(prob.g)
            success, gnorm = self.ls.search(prob, m0, p, k, self.max_trial, self.counts, gnorm)
            self.steps.append(self.ls.stp)
            if not success:
                break
            f = prob.get_func()
            self.func.append(f)
            if k > 0:
                rate = (self.func[k] - self.func[k + 1]) / self.func[k]
            k += 1
        return prob


class Nlcg(_Solver):
    """Non-linear conjugate gradient (nlsolver.cpp:815-945); method 0
    Fletcher-Reeves, 1 Polak-Ribiere, 2 Polak-Ribiere+."""

    def __init__(self, niter: int, max_trial: int = 10, threshold: float = 0.0, ls=None, method: int = 0):
        super().__init__(niter, max_trial, threshold, ls)
        self.method = method if method in (1, 2) else 0

    def run(self, prob: Problem) -> Problem:
        be = prob.be
        if not self._start(prob):
            return prob
        m0 = be.copy(prob.m)
        p = be.copy(prob.g)
        g0 = None
        beta, k, rate, gnorm, gnorm0, f = 0.0, 0, 1.0, 999.0, -1.0, self.func[0]
        success = True
        while k < self.niter and rate > self.threshold and gnorm > ZERO and f > ZERO and success:
            if self.ls.flag_g or k == 0:
                prob.grad()
                self.counts["geval"] += 1
                gnorm = be.norm(prob.g)
            if k > 0:
                if self.method == 0:
                    beta = gnorm * gnorm / (gnorm0 * gnorm0)
                elif self.method == 1:
                    beta = (gnorm * gnorm - be.dot(prob.g, g0)) / (gnorm0 * gnorm0)
                else:
                    beta = max(0.0, (gnorm * gnorm - be.dot(prob.g, g0)) / (gnorm0 * gnorm0))
            p = beta * p - prob.g  # scaleAdd(g, beta, -1)
            if be.dot(p, prob.g) >= 0:
                break
            if k > 0:
                m0 = be.copy(prob.m)
            if self.method > 0:
                g0 = be.copy(prob.g)
            gnorm0 = gnorm
            success, gnorm = self.ls.search(prob, m0, p, k, self.max_trial, self.counts, gnorm)
            self.steps.append(self.ls.stp)
            if not success:
                break
            f = prob.get_func()
            self.func.append(f)
            if k > 0:
                rate = (self.func[k] - self.func[k + 1]) / self.func[k]
            k += 1
        return prob


class Nlsd(Nlcg):
    """Non-linear steepest descent: the NLCG loop with beta = 0."""

    def __init__(self, niter: int, max_trial: int = 10, threshold: float = 0.0, ls=None):
        super().__init__(niter, max_trial, threshold, ls, method=0)

    def run(self, prob: Problem) -> Problem:
        be = prob.be
        if not self._start(prob):
            return prob
        m0 = be.copy(prob.m)
        k, rate, gnorm, f = 0, 1.0, 999.0, self.func[0]
        success = True
        while k < self.niter and rate > self.threshold and gnorm > ZERO and f > ZERO and success:
            if self.ls.flag_g or k == 0:
                prob.grad()
                self.counts["geval"] += 1
                gnorm = be.norm(prob.g)
            p = -1.0 * prob.g
            if k > 0:
                m0 = be.copy(prob.m)
            success, gnorm = self.ls.search(prob, m0, p, k, self.max_trial, self.counts, gnorm)
            self.steps.append(self.ls.stp)
            if not success:
                break
            f = prob.get_func()
            self.func.append(f)
            if k > 0:
                rate = (self.func[k] - self.func[k + 1]) / self.func[k]
            k += 1
        return prob


def make_line_search(name: str = "regular_wolfe", c1: float = 1e-4, c2: float = 0.9, a0: float = 1.0,
                     a1: float = 0.0, step_max: float = 1e6, version: bool = False):
    """The reference FWI program's choice (fwi3d.cpp: par.lsearch)."""
    if name == "weak_wolfe":
        return WeakWolfe(c1, a0, a1, version)
    if name == "regular_wolfe":
        return RegularWolfe(c1, c2, a0, a1, step_max, version)
    raise ValueError(f"line search {name!r} is not implemented (weak_wolfe, regular_wolfe)")


def make_solver(name: str, niter: int, max_trial: int = 10, threshold: float = 0.0, ls=None, m: int = 5,
                method: int = 0, h0=None):
    """The reference FWI program's choice (fwi3d.cpp: par.nlsolver)."""
    if name == "nlsd":
        return Nlsd(niter, max_trial, threshold, ls)
    if name == "nlcg":
        return Nlcg(niter, max_trial, threshold, ls, method)
    if name == "lbfgs":
        return Lbfgs(niter, max_trial, threshold, ls, h0, m)
    raise ValueError(f"solver {name!r} is not implemented (nlsd, nlcg, lbfgs)")
