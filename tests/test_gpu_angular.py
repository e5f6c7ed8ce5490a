"""Angular on the device against the oracle (through the C ABI): spline
tables (one and two species) and analytic tables.

Tolerances:
  FP64  forces, energy, stress, F rows   |Δ| ≤ 1e-9·(1 + |x|); objective 1e-9 relative
  FP32  forces                           |Δ| ≤ 2e-5·max|F|;    objective 1e-4 relative
  Jacobian (FP64 central differences, h = 1e-5, the reference's method for
  spline tables, against the oracle's own central differences)
                                         |ΔJ| ≤ 1e-5·max|J column| + 1e-7
"""
import numpy as np
import pytest

from forcesmith_b200.abi import FS_FAMILY_ANGULAR, Model, Table
from oracle import api as O
from tests.helpers import label, small_ternary

pytestmark = pytest.mark.gpu


def spline_model(nt, scale=1.0, nk=10):
    np_ = nt * (nt + 1) // 2
    r = np.linspace(1.8, 4.6, nk)
    tabs = []
    for s in range(np_):
        tabs.append(Table.spline(1.8, 4.6, scale * 0.3 * (np.exp(-2 * (r - 2.6)) - 2 * np.exp(-(r - 2.6)))
                                 * (1 - (r / 4.6) ** 4) * (1 + 0.05 * s)))
    for s in range(np_):
        tabs.append(Table.spline(1.8, 4.6, scale * np.exp(-1.1 * (r - 2.0)) * (1 - (r / 4.6) ** 3) * (1 + 0.03 * s)))
    c = np.linspace(-1.0, 1.0, 9)
    for t in range(nt):
        tabs.append(Table.spline(-1.0, 1.0, scale * 0.4 * (c + 1.0 / 3.0) ** 2 * (1 + 0.1 * t)))
    return Model(FS_FAMILY_ANGULAR, nt, tabs)


def analytic_model(scale=1.0):
    return Model(FS_FAMILY_ANGULAR, 1, [
        Table.analytic("morse", [0.3 * scale, 1.4, 2.7], 1.5, 4.5),
        Table.analytic("exp_decay", [1.0 * scale, 0.9], 1.5, 4.5),
        Table.analytic("harmonic", [0.5 * scale, -1.0 / 3.0], -1.0, 1.0)])


def _pair(ds, model, precision):
    from forcesmith_b200.gpu import GpuSession
    g = GpuSession(0, precision)
    g.upload(ds)
    g.set_model(model)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model)
    return g, o


def _close(a, b, rel, what):
    err = np.max(np.abs(np.asarray(a) - np.asarray(b)) / (1.0 + np.abs(np.asarray(b))))
    assert err <= rel, f"{what}: {err:.3e}"


@pytest.fixture(scope="module", params=["spline1", "spline2", "analytic"])
def case(request):
    ds = small_ternary(3, 40, seed=61)
    if request.param == "spline1":
        ds.type[:] = 0
        true, start = spline_model(1), spline_model(1, 1.03)
    elif request.param == "spline2":
        ds.type[:] = ds.type % 2
        true, start = spline_model(2), spline_model(2, 1.03)
    else:
        ds.type[:] = 0
        true, start = analytic_model(), analytic_model(1.04)
    return label(ds, true, O.Oracle, 1.0, 0.2), start


def test_angular_residual_fp64(case):
    ds, start = case
    g, o = _pair(ds, start, "fp64")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    _close(rg["forces"], ro["forces"], 1e-9, "forces")
    _close(rg["energy"], ro["energy"], 1e-9, "energy")
    _close(rg["stress"], ro["stress"], 1e-9, "stress")
    _close(rg["F"], ro["F"], 1e-9, "F")
    assert abs(rg["obj"] - ro["obj"]) <= 1e-9 * ro["obj"]


def test_angular_residual_fp32(case):
    ds, start = case
    g, o = _pair(ds, start, "fp32")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    assert np.max(np.abs(rg["forces"] - ro["forces"])) <= 2e-5 * np.max(np.abs(ro["forces"]))
    assert abs(rg["obj"] - ro["obj"]) <= 1e-4 * ro["obj"]


def test_angular_jacobian_central_differences(case):
    ds, start = case
    g, o = _pair(ds, start, "fp64")
    res = g.jacobian(1.0, 0.2)
    Jf = o.jacobian_fd(1.0, 0.2)
    assert res["J"].shape == Jf.shape
    colmax = np.abs(Jf).max(axis=0)
    bar = 1e-5 * colmax + 1e-7
    ratio = np.abs(res["J"] - Jf) / bar
    r, c = np.unravel_index(np.argmax(ratio), ratio.shape)
    assert ratio.max() <= 1.0, (ratio.max(), r, c, res["J"][r, c], Jf[r, c])
    F = o.eval(1.0, 0.2)["F"]
    _, Jtr = O.normal_equations(Jf, F)
    assert np.max(np.abs(res["Jtr"] - Jtr)) <= 1e-5 * np.max(np.abs(Jtr))
