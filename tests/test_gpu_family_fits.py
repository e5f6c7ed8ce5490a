"""End-to-end fits on the §8(f) families through the solver layer
(solvers.py → C ABI → device): LM on Tersoff and Angular (FP64 contexts,
the device's central-difference Jacobian), and the one-shot normal-equations
solver on ACSF with a linear head (the reference's lsq for such models).

Bars: the fitted objective falls below the stated fraction of the start.
"""
import numpy as np
import pytest

from forcesmith_b200 import solvers, synth
from oracle import api as O
from tests.helpers import label
from tests.test_gpu_three_body_edges import models

pytestmark = pytest.mark.gpu


def _session(ds, m):
    from forcesmith_b200.gpu import GpuSession
    g = GpuSession(0, "fp64")
    g.upload(ds)
    g.set_model(m)
    return g


@pytest.mark.parametrize("which,scale,frac", [("tersoff", 1.03, 1e-3), ("angular", 1.05, 1e-2)])
def test_lm_fit_recovers_labels(which, scale, frac):
    true = models()[which]
    ds = label(synth.diamond(3, cells=(2,), seed=91), true, O.Oracle, 1.0, 0.0)
    start = true.with_values(true.free_values() * scale)
    g = _session(ds, start)
    x0 = g.gather_params()
    o0 = g.eval(1.0, 0.0, want=("obj",))["obj"]
    status, x, info = solvers.LMSolver(max_iter=40).minimize(g, x0)
    o1 = g.eval(1.0, 0.0, want=("obj",))["obj"]
    assert o0 > 0 and o1 <= frac * o0, (which, o0, o1, info["iterations"])


def test_normal_equations_fit_acsf():
    true = models()["acsf"]
    ds = label(synth.diamond(3, cells=(2,), seed=93), true, O.Oracle, 1.0, 0.1)
    start = true.with_values(true.free_values() * np.linspace(0.8, 1.2, true.free_values().size))
    g = _session(ds, start)
    o0 = g.eval(1.0, 0.1, want=("obj",))["obj"]
    _, x, _ = solvers.NormalEquationsSolver().minimize(g, g.gather_params(), w_e=1.0, w_s=0.1)
    o1 = g.eval(1.0, 0.1, want=("obj",))["obj"]
    assert o1 <= 1e-8 * o0, (o0, o1)
    np.testing.assert_allclose(x, true.free_values(), rtol=1e-4, atol=1e-6)
