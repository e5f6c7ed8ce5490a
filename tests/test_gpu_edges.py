"""Edge cases of the residual and Jacobian against the oracle, the inputs
the reference's tests exercise: a ragged batch with an isolated atom (no
neighbours), a dimer, a triclinic box with unwrapped positions and regular
configurations; models with fixed knots (one table entirely fixed, so it
takes no columns).  Bars as in test_gpu_parity.py: FP64 1e-9·(1 + |x|),
Jacobian 1e-9·(1 + |J|) against the oracle's analytic Jacobian; FP32 forces
2e-5·max|F|, J columns 1e-4·max|column|."""
import numpy as np
import pytest

from forcesmith_b200.abi import Model, Table
from oracle import api as O
from tests.helpers import cluster, concat, label, small_ternary, ternary_models

pytestmark = pytest.mark.gpu


def ragged():
    iso = cluster([[1.0, 1.0, 1.0]], 30.0, types=[2])
    dimer = cluster([[0.0, 0.0, 0.0], [2.6, 0.3, 0.0]], 25.0, types=[0, 1])
    rng = np.random.default_rng(3)
    tri = cluster(rng.uniform(-4, 16, (36, 3)), 12.0, types=rng.integers(0, 3, 36))
    tri.box9[0] = [12.0, 6.0, 1.0, 0.0, 10.39, 0.5, 0.0, 0.0, 11.0]
    regular = small_ternary(2, 48, seed=41)
    return concat(iso, dimer, tri, regular.subset([0]), regular.subset([1]))


def fixed_model():
    _, start = ternary_models(20)
    tabs = []
    for k, t in enumerate(start.tables):
        fx = np.zeros(t.values.size, np.uint8)
        if k == 2:
            fx[:] = 1  # a whole pair table fixed
        elif k % 3 == 0:
            fx[::4] = 1  # every fourth knot fixed
        tabs.append(Table.spline(t.rmin, t.rmax, t.values, fixed=fx))
    return Model(start.family, start.ntypes, tabs)


def _sessions(ds, model, precision):
    from forcesmith_b200.gpu import GpuSession
    true, _ = ternary_models(20)
    ds = label(ds, true, O.Oracle, 1.0, 0.1)
    g = GpuSession(0, precision)
    g.upload(ds)
    g.set_model(model)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model)
    return g, o


def _close(a, b, tol, what):
    err = np.max(np.abs(np.asarray(a) - np.asarray(b)) / (1.0 + np.abs(b)))
    assert err <= tol, f"{what}: {err:.3e}"


@pytest.mark.parametrize("which", ["ragged", "fixed"])
def test_residual_and_jacobian_fp64(which):
    ds = ragged() if which == "ragged" else small_ternary(3, 48, seed=9)
    model = ternary_models(20)[1] if which == "ragged" else fixed_model()
    g, o = _sessions(ds, model, "fp64")
    assert g.D == o.D
    a, b = g.eval(1.0, 0.1), o.eval(1.0, 0.1)
    for k in ("forces", "energy", "stress", "F", "limit"):
        _close(a[k], b[k], 1e-9, k)
    J = g.jacobian(1.0, 0.1)["J"]
    Jo = o.jacobian_analytic(1.0, 0.1)
    assert J.shape == Jo.shape
    assert np.all(np.abs(J - Jo) <= 1e-9 * (1.0 + np.abs(Jo)))
    if which == "ragged":
        # the isolated atom: zero force rows in F's reference row order
        assert np.all(a["forces"][0] == 0.0)


@pytest.mark.parametrize("which", ["ragged", "fixed"])
def test_residual_and_jacobian_fp32(which):
    ds = ragged() if which == "ragged" else small_ternary(3, 48, seed=9)
    model = ternary_models(20)[1] if which == "ragged" else fixed_model()
    g, o = _sessions(ds, model, "fp32")
    a, b = g.eval(1.0, 0.1), o.eval(1.0, 0.1)
    assert np.max(np.abs(a["forces"] - b["forces"])) <= 2e-5 * np.max(np.abs(b["forces"]))
    J = g.jacobian(1.0, 0.1)["J"]
    Jo = o.jacobian_analytic(1.0, 0.1)
    scale = np.max(np.abs(Jo), axis=0)
    assert np.all(np.abs(J - Jo) <= 1e-4 * scale[None, :] + 1e-12)


def test_fixed_knots_layout():
    g, o = _sessions(small_ternary(1, 48, seed=9), fixed_model(), "fp64")
    assert g.D == o.D < 240
    np.testing.assert_array_equal(g.gather_params(), o.gather_params())
