"""Host-side logic of the step consumers (forcesmith_b200/solvers.py), run on
CPU against the oracle behind the same step interface."""
import numpy as np
import pytest

from forcesmith_b200 import solvers
from oracle import api as O
from tests.de_rule import de_init_population, de_trials, urand
from tests.helpers import label, small_ternary, ternary_models
from tests.oracle_session import OracleStepSession


@pytest.fixture(scope="module")
def problem():
    true, start = ternary_models(8)
    ds = label(small_ternary(3, 32, seed=11), true, O.Oracle, 1.0, 0.0)
    return ds, true, start


def _session(ds, model):
    s = OracleStepSession()
    s.upload(ds)
    s.set_model(model)
    return s


def test_de_box_rule():
    # solver.cpp:118-124: finite bounds kept; otherwise x ∓ max(2|x|, 5e-4)
    x = np.array([1.0, -3.0, 0.0, 1e-5])
    lo = np.array([0.5, -np.inf, -np.inf, -np.inf])
    hi = np.array([np.inf, 2.0, np.inf, np.inf])
    lb, ub = solvers.de_box(x, lo, hi)
    np.testing.assert_array_equal(lb, [0.5, -9.0, -5e-4, 1e-5 - 5e-4])
    np.testing.assert_array_equal(ub, [3.0, 2.0, 5e-4, 1e-5 + 5e-4])


def test_de_rule_restatement_properties():
    u = np.array([urand(42, g, i, d) for g in range(3) for i in range(20) for d in range(20)])
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.05 and len(np.unique(u)) == u.size
    lo, hi = np.full(6, -1.0), np.full(6, 2.0)
    pop = de_init_population(9, lo, hi, np.array([5.0, 0, 0, 0, 0, -7.0]), 10)
    assert pop[0, 0] == 2.0 and pop[0, 5] == -1.0
    assert np.all(pop >= lo) and np.all(pop <= hi)
    t = de_trials(9, 0, pop, lo, hi, 0.65, 0.0)  # CR = 0: exactly one coordinate crosses
    assert np.all((t != pop).sum(axis=1) <= 1)
    assert np.all(t >= lo) and np.all(t <= hi)


def test_lm_converges_on_oracle(problem):
    ds, _, start = problem
    s = _session(ds, start)
    x = s.gather_params()
    o0 = s.eval(1.0, 0.0, want=("obj",))["obj"]
    st, xf, info = solvers.LMSolver(max_iter=12).minimize(s, x)
    assert st in (1, 2, 3, 5)
    assert info["obj"][-1] < 1e-3 * o0
    assert all(b <= a for a, b in zip(info["obj"], info["obj"][1:]))
    assert s.eval(1.0, 0.0, want=("obj",))["obj"] == pytest.approx(info["obj"][-1], rel=1e-12)


def test_dogleg_converges_on_oracle(problem):
    ds, _, start = problem
    s = _session(ds, start)
    x = s.gather_params()
    o0 = s.eval(1.0, 0.0, want=("obj",))["obj"]
    st, xf, info = solvers.HybridSolver(max_iter=12).minimize(s, x)
    assert info["obj"][-1] < 1e-3 * o0
    assert all(b <= a for a, b in zip(info["obj"], info["obj"][1:]))


def test_normal_equations_step(problem):
    ds, _, start = problem
    s = _session(ds, start)
    x = s.gather_params()
    F = s.eval(1.0, 0.0, want=("F",))["F"]
    J = s.jacobian_analytic(1.0, 0.0)
    A = J.T @ J
    lam = 1e-8 * max(np.mean(np.diag(A)), 1.0)
    want = x - np.linalg.solve(A + lam * np.eye(x.size), J.T @ F)
    _, got, _ = solvers.NormalEquationsSolver().minimize(s, x)
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-9)
    assert solvers.NormalEquationsSolver().one_shot() and solvers.DESolver().honors_bounds()
