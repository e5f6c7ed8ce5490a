"""The Al99 LM-fit fixture on CPU: the pin of its labels and the
oracle-driven LM fit that the device fit is compared with."""
import numpy as np

from forcesmith_b200 import solvers
from tests.al99 import load
from tests.oracle_session import OracleStepSession


def test_label_potential_pin():
    # Al99 (Phys. Rev. B 59, 3393): cohesive energy 3.36 eV at a0 = 4.05 Å
    _, _, e = load()
    assert abs(e - (-3.36)) < 1e-5


def test_oracle_lm_fit_reduces_objective():
    ds, start, _ = load()
    s = OracleStepSession()
    s.upload(ds)
    s.set_model(start)
    assert s.D == 45 and s.residual_count(0.0) == 6520
    x0 = s.gather_params()
    o0 = s.eval(1.0, 0.0, want=("obj",))["obj"]
    _, x, info = solvers.LMSolver(max_iter=200).minimize(s, x0)
    # 15 knots cannot reproduce the 10,000-knot label potential, and LM stops
    # at a kink of the makima objective (|·| weights in the slopes): from 201
    # to about 64
    assert info["obj"][-1] < 0.5 * o0
    assert np.all(np.diff(info["obj"]) <= 0)
