"""ADP on the device (ADPForceCalculator, src/force/adp_force.cpp): residual
and exact parameter Jacobian (forward mode, one column per CTA row) for
spline and analytic tables, in FP64 and FP32, against the oracle.

The reference has no analytic ADP Jacobian for spline tables; its method is
central differences of the residual (fd_jacobian.hpp:37-49).  J_fd below is
that, over the oracle's FP64 residual, with a step of 1e-7 instead of the
reference's 1e-5: the spline model's smallest quadrupole knots are ~1e-4,
where a 1e-5 step is a 10 % change and the makima weights make the central
difference itself off by up to 3 % of the column (the 1e-7 step agrees with
the device's forward-mode J to 5e-7).  Bars:
  FP64   |J − J_fd| ≤ 1e-5·|J_fd| + 1e-8 + 1e-5·max|J_fd column| (the
         step's rounding noise is ~3e-6 of a column); Jᵀr 1e-6 of its
         largest entry
  FP32   |J − J_fd| ≤ 1e-4·max|J_fd column|
Residual: FP64 1e-9·(1 + |x|), FP32 forces 2e-5·max|F|.
"""
import numpy as np
import pytest

from forcesmith_b200.abi import FS_FAMILY_ADP, Model, Table
from oracle import api as O
from tests.helpers import adp_spline_model, label, small_ternary

pytestmark = pytest.mark.gpu

RC = 5.5


def adp_analytic_model(nt=2, emb_hi=1e6):
    np_ = nt * (nt + 1) // 2
    pairs = [Table.analytic("morse", [0.25 + 0.03 * k, 1.5, 2.7 + 0.05 * k], 0.5, RC) for k in range(np_)]
    dens = [Table.analytic("exp_decay", [2.0 + 0.5 * k, 1.2], 0.5, RC) for k in range(nt)]
    emb = [Table.analytic("sqrt", [-1.0 - 0.2 * k, 1.0], 0.0, emb_hi) for k in range(nt)]
    dip = [Table.analytic("mexp_decay", [0.05 + 0.01 * k, 1.0, 2.5], 0.5, RC) for k in range(np_)]
    quad = [Table.analytic("exp_decay", [0.3 + 0.05 * k, 1.6], 0.5, RC) for k in range(np_)]
    return Model(FS_FAMILY_ADP, nt, pairs + dens + emb + dip + quad)


def _case(model):
    ds = small_ternary(3, 32, seed=41)
    ds.type[:] = ds.type % 2
    ds = label(ds, model.with_values(model.free_values() * 1.02), O.Oracle, 1.0, 0.1)
    return ds


def _pair(ds, model, precision):
    from forcesmith_b200.gpu import GpuSession
    g = GpuSession(0, precision)
    g.upload(ds)
    g.set_model(model)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model)
    return g, o


def central_differences(o, h):
    """J by central differences of the oracle's residual, step h."""
    x0 = o.gather_params()
    cols = []
    for c in range(x0.size):
        xp, xm = x0.copy(), x0.copy()
        xp[c] += h
        xm[c] -= h
        o.set_params(xp)
        fp = o.eval(1.0, 0.1, want=("F",))["F"]
        o.set_params(xm)
        fm = o.eval(1.0, 0.1, want=("F",))["F"]
        cols.append((fp - fm) / (2 * h))
    o.set_params(x0)
    return np.stack(cols, axis=1)


MODELS = {"spline": adp_spline_model, "analytic": adp_analytic_model,
          "analytic_clamped": lambda: adp_analytic_model(emb_hi=1.0)}


@pytest.mark.parametrize("name", list(MODELS))
def test_adp_residual(name):
    model = MODELS[name]()
    ds = _case(model)
    for precision in ("fp64", "fp32"):
        g, o = _pair(ds, model, precision)
        a, b = g.eval(1.0, 0.1), o.eval(1.0, 0.1)
        if precision == "fp64":
            for k in ("forces", "energy", "stress", "F", "limit"):
                err = np.max(np.abs(a[k] - b[k]) / (1.0 + np.abs(b[k])))
                assert err <= 1e-9, (k, err)
        else:
            assert np.max(np.abs(a["forces"] - b["forces"])) <= 2e-5 * np.max(np.abs(b["forces"]))


def test_clamped_model_has_live_limit_rows():
    model = adp_analytic_model(emb_hi=1.0)
    _, o = _pair(_case(model), model, "fp64")
    assert np.any(o.eval(1.0, 0.1)["limit"] > 0)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", list(MODELS))
def test_adp_jacobian_exact(name, precision):
    model = MODELS[name]()
    ds = _case(model)
    g, o = _pair(ds, model, precision)
    res = g.jacobian(1.0, 0.1)
    Jf = central_differences(o, 1e-7)
    assert res["J"].shape == Jf.shape
    colmax = np.abs(Jf).max(axis=0)
    if precision == "fp64":
        bound = 1e-5 * np.abs(Jf) + 1e-8 + 1e-5 * colmax[None, :]
        assert np.all(np.abs(res["J"] - Jf) <= bound), np.max(np.abs(res["J"] - Jf) / bound)
        F = o.eval(1.0, 0.1)["F"]
        Jtr = Jf.T @ F
        assert np.max(np.abs(res["Jtr"] - Jtr)) <= 1e-6 * np.max(np.abs(Jtr))
        JtJ = res["J"].T @ res["J"]
        assert np.allclose(res["JtJ"], JtJ, rtol=1e-9, atol=1e-12 * np.abs(JtJ).max())
    else:
        assert np.max(np.abs(res["J"] - Jf) / (colmax[None, :] + 1e-30)) <= 1e-4
