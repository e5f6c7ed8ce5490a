"""The evaluate report from the device path against the oracle's (FP64:
energies, stresses, forces and per-configuration sums within 1e-9·(1 + |x|);
total within 1e-9 relative)."""
import numpy as np
import pytest

from forcesmith_b200.evaluate import evaluate_report
from oracle import api as O
from tests.helpers import label, small_ternary, ternary_models

pytestmark = pytest.mark.gpu


def test_evaluate_report_matches_oracle():
    from forcesmith_b200.gpu import GpuSession
    true, start = ternary_models(20)
    ds = label(small_ternary(4, 36, seed=12), true, O.Oracle, 1.0, 0.1)
    reps = []
    for s in (GpuSession(0, "fp64"), O.Oracle()):
        s.upload(ds)
        s.set_model(start)
        reps.append(evaluate_report(s, ds, 1.0, 0.1))
    g, o = reps
    assert abs(g["total_sumsq"] - o["total_sumsq"]) <= 1e-9 * o["total_sumsq"]
    for a, b in zip(g["configs"], o["configs"]):
        for k in ("calc_energy", "limit", "sumsq"):
            assert abs(a[k] - b[k]) <= 1e-9 * (1 + abs(b[k]))
        assert np.allclose(a["calc_stress"], b["calc_stress"], rtol=1e-9, atol=1e-9)
        fa = np.array([x["calc_force"] for x in a["atoms"]])
        fb = np.array([x["calc_force"] for x in b["atoms"]])
        assert np.all(np.abs(fa - fb) <= 1e-9 * (1 + np.abs(fb)))
