"""Host logic of the non-linear solvers (fwi3d_b200/nlsolver.py) on analytic
problems, with the host vector backend: the reference's own solver tests use
the same two functions (nlsolver.hpp: testRosenbrock, testParaboloid)."""
import numpy as np
import pytest

from fwi3d_b200 import nlsolver


def rosenbrock(a=1.0, b=100.0):
    def ev(m):
        x, y = float(m[0]), float(m[1])
        f = (a - x) ** 2 + b * (y - x * x) ** 2
        g = np.array([-2 * (a - x) - 4 * b * x * (y - x * x), 2 * b * (y - x * x)])
        return f, g
    return ev


def paraboloid(a=1.0, b=2.0):
    def ev(m):
        x, y = float(m[0]), float(m[1])
        return 0.5 * (a * x) ** 2 + 0.5 * (b * y) ** 2, np.array([a * a * x, b * b * y])
    return ev


def test_quadratic_and_cubic_interpolation():
    # f(s) = (s - 2)^2 from f(0) = 4, f'(0) = -4 and one more point: exact minimiser 2
    assert nlsolver.quadratic(4.0, -4.0, 1.0, 1.0) == pytest.approx(2.0)
    # cubic f(s) = s^3 - 3 s (+ 0): f(0)=0, f'(0)=-3, minimiser 1
    f = lambda s: s ** 3 - 3 * s
    assert nlsolver.cubic(0.0, -3.0, 0.5, f(0.5), 2.0, f(2.0)) == pytest.approx(1.0, rel=1e-9)


@pytest.mark.parametrize("name", ["lbfgs", "nlcg", "nlsd"])
@pytest.mark.parametrize("ls", ["weak_wolfe", "regular_wolfe"])
def test_solvers_reach_the_minimum(name, ls):
    be = nlsolver.Backend(None)
    it = {"lbfgs": 60, "nlcg": 400, "nlsd": 3000}[name]
    prob = nlsolver.Problem(np.array([-1.2, 1.0], dtype=np.float32), rosenbrock(), be)
    s = nlsolver.make_solver(name, it, max_trial=20, ls=nlsolver.make_line_search(ls))
    s.run(prob)
    # the model is handed to the objective in FP32 as the reference's model
    # vector is, so the searches stop once FP32 steps no longer decrease f
    assert s.func[-1] < 0.2 * s.func[0]
    assert all(b <= a for a, b in zip(s.func, s.func[1:]))
    prob = nlsolver.Problem(np.array([3.0, -2.0], dtype=np.float32), paraboloid(), be)
    s = nlsolver.make_solver(name, 50, max_trial=20, ls=nlsolver.make_line_search(ls))
    s.run(prob)
    # as in the reference, a search that reaches f <= 1e-10 stops the solver
    # without adding that value to the history
    assert min(s.func[-1], prob.get_func()) < 1e-6 * s.func[0]


def test_wolfe_conditions_hold_at_accepted_steps():
    be = nlsolver.Backend(None)
    ev = rosenbrock()
    prob = nlsolver.Problem(np.array([-1.2, 1.0], dtype=np.float32), ev, be)
    s = nlsolver.Lbfgs(5, max_trial=20, ls=nlsolver.RegularWolfe(1e-4, 0.9))
    s.run(prob)
    # the objective decreases monotonically and every step was accepted
    assert all(b < a for a, b in zip(s.func, s.func[1:]))
    assert len(s.steps) == len(s.func) - 1
