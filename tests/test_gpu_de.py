"""Device differential evolution and the device-driven solvers, against the
oracle.

  one generation     bit-exact against a restatement of the trial rule
                     (counter-hash RNG, DE/rand/1/bin, clamp, greedy ≤)
                     with objectives from the oracle (relative 1e-9)
  population objs    the device's kept objectives = oracle objectives of the
                     device population, relative 1e-9 (FP64 context)
  graph replay       identical populations with and without the CUDA graph
  bounds             every member inside de_box
  LM / dogleg / lsq  final objective within 10 % of the oracle-driven run of
                     the same solver (the reference's integration tests use
                     the same 10 % bar, test_integration.cpp:313,501,579)
"""
import numpy as np
import pytest

from forcesmith_b200 import solvers, synth
from oracle import api as O
from tests.helpers import label, small_ternary, ternary_models
from tests.de_rule import de_init_population, de_trials

pytestmark = pytest.mark.gpu


def _gpu(precision="fp64"):
    from forcesmith_b200.gpu import GpuSession
    return GpuSession(0, precision)


@pytest.fixture(scope="module")
def problem():
    true, start = ternary_models(12)
    ds = label(small_ternary(4, 40, seed=5), true, O.Oracle, 1.0, 0.0)
    return ds, true, start


def _sessions(ds, model, precision="fp64"):
    g = _gpu(precision)
    g.upload(ds)
    g.set_model(model)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model)
    return g, o


def test_de_first_generation_exact(problem):
    ds, _, start = problem
    g, o = _sessions(ds, start)
    x0 = g.gather_params()
    lb, ub = solvers.de_box(x0)
    NP, F, CR, seed = 24, 0.65, 0.5, 1234
    g.de_init(lb, ub, x0=x0, NP=NP, mutation=F, crossover=CR, seed=seed)
    pop0, obj0 = g.de_population()
    ref0 = de_init_population(seed, lb, ub, x0, NP)
    assert np.array_equal(pop0, ref0)
    oo0 = o.eval_population(pop0, 1.0, 0.0)
    np.testing.assert_allclose(obj0, oo0, rtol=1e-9)
    g.de_run(1, use_graph=False)
    pop1, obj1 = g.de_population()
    trial = de_trials(seed, 0, pop0, lb, ub, F, CR)
    tobj = o.eval_population(trial, 1.0, 0.0)
    take = tobj <= obj0  # within rounding the device and oracle agree; check both sides
    close = np.abs(tobj - obj0) <= 1e-9 * np.abs(obj0)
    for i in range(NP):
        if close[i]:
            assert np.array_equal(pop1[i], trial[i]) or np.array_equal(pop1[i], pop0[i])
        else:
            assert np.array_equal(pop1[i], trial[i] if take[i] else pop0[i]), i
    np.testing.assert_allclose(obj1, o.eval_population(pop1, 1.0, 0.0), rtol=1e-9)


def test_de_graph_replay_matches_stream(problem):
    ds, _, start = problem
    out = []
    for use_graph in (False, True):
        g = _gpu("fp64")
        g.upload(ds)
        g.set_model(start)
        x = g.gather_params()
        lb, ub = solvers.de_box(x)
        g.de_init(lb, ub, x0=x, NP=32, seed=7)
        best, xb, hist = g.de_run(6, use_graph=use_graph, history=True)
        pop, obj = g.de_population()
        assert np.all(pop >= lb) and np.all(pop <= ub)
        assert np.all(np.diff(hist) <= 0.0), "best objective must not increase"
        out.append((pop, obj, best, xb))
        g.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]


def test_de_solver_reduces_objective(problem):
    ds, _, start = problem
    g = _gpu("fp32")
    g.upload(ds)
    g.set_model(start)
    x = g.gather_params()
    o0 = g.eval(1.0, 0.0, want=("obj",))["obj"]
    lo, hi = x - 0.1 * np.abs(x) - 1e-3, x + 0.1 * np.abs(x) + 1e-3  # finite bounds are kept
    st, xb, info = solvers.DESolver(NP_factor=2, max_generations=40, seed=3).minimize(g, x, lo, hi,
                                                                                      history=True)
    np.testing.assert_array_equal(info["lower"], lo)
    assert st == 0
    assert info["obj"] <= o0
    assert info["history"][-1] < info["history"][0]
    lb, ub = info["lower"], info["upper"]
    assert np.all(xb >= lb) and np.all(xb <= ub)


def _oracle_step_session(ds, model):
    from tests.oracle_session import OracleStepSession
    s = OracleStepSession()
    s.upload(ds)
    s.set_model(model)
    return s


@pytest.mark.parametrize("make", [lambda: solvers.LMSolver(max_iter=15),
                                  lambda: solvers.HybridSolver(max_iter=15)],
                         ids=["lm", "dogleg"])
def test_device_solver_vs_oracle_driven(problem, make):
    ds, _, start = problem
    g = _gpu("fp64")
    g.upload(ds)
    g.set_model(start)
    x = g.gather_params()
    o0 = g.eval(1.0, 0.0, want=("obj",))["obj"]
    _, xg, ig = make().minimize(g, x)
    og = g.eval(1.0, 0.0, want=("obj",))["obj"]
    s = _oracle_step_session(ds, start)
    _, xo, io = make().minimize(s, x)
    oo = s.eval(1.0, 0.0, want=("obj",))["obj"]
    assert og < 1e-4 * o0
    floor = 1e-9 * o0  # both runs converge to ~0 on exactly-representable labels
    assert og <= 1.1 * oo + floor and oo <= 1.1 * og + floor


def test_normal_equations_solver_matches_oracle(problem):
    ds, _, start = problem
    g = _gpu("fp64")
    g.upload(ds)
    g.set_model(start)
    x = g.gather_params()
    _, xg, _ = solvers.NormalEquationsSolver().minimize(g, x)
    s = _oracle_step_session(ds, start)
    _, xo, _ = solvers.NormalEquationsSolver().minimize(s, x)
    np.testing.assert_allclose(xg, xo, rtol=1e-7, atol=1e-9 * np.max(np.abs(x)))
