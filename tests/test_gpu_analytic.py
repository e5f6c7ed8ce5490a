"""Analytic radial tables on the device (the reference's AnalyticForm
potentials, include/forcesmith/potentials/analytic_potential.hpp), against
the oracle.

  FP64 residual   |Δ| ≤ 1e-9·(1 + |x|) (forces, energies, stress, F rows)
  FP32 residual   forces 2e-5·max|F|, objective 1e-4 relative
  Jacobian        the device's central differences (the reference's method
                  for these tables, fd_jacobian.hpp:37-49, FP64 contexts)
                  against the oracle's analytic parameter Jacobian:
                  |Δ| ≤ 1e-5·max|column| + 1e-8 (test_param_jacobian.cpp:70)
"""
import numpy as np
import pytest

from forcesmith_b200.abi import FS_ERR_UNSUPPORTED, FS_FAMILY_EAM, FS_FAMILY_PAIR, FsError, Model, Table
from oracle import api as O
from tests.helpers import label, small_ternary, ternary_models

pytestmark = pytest.mark.gpu

RC = 5.5


def pair_model():
    return Model(FS_FAMILY_PAIR, 3, [
        Table.analytic("lj", [0.2, 2.5], 0.5, RC),
        Table.analytic("morse", [0.3, 1.5, 2.8], 0.5, RC),
        Table.analytic("buckingham", [800.0, 0.3, 12.0], 0.5, RC),
        Table.analytic("born", [0.5, 0.35, 2.0, 8.0, 6.0], 0.5, RC),
        Table.analytic("mexp_decay", [0.4, 1.8, 2.6], 0.5, RC),
        Table.analytic("exp_plus", [50.0, 3.0, -0.01], 0.5, RC),
    ])


def eam_model(spline_pairs=False):
    pairs = ternary_models(20)[1].tables[:6] if spline_pairs else [
        Table.analytic("morse", [0.25 + 0.05 * k, 1.4 + 0.05 * k, 2.7 + 0.05 * k], 0.5, RC) for k in range(6)]
    dens = [Table.analytic("exp_decay", [3.0 + k, 1.2 + 0.1 * k], 0.5, RC) for k in range(3)]
    emb = [Table.analytic("sqrt", [-1.0 - 0.2 * k, 1.0], 0.0, 1e6) for k in range(3)]
    return Model(FS_FAMILY_EAM, 3, pairs + dens + emb)


MODELS = {"pair": pair_model, "eam": eam_model, "eam_mixed": lambda: eam_model(True)}


def _sessions(model, precision):
    from forcesmith_b200.gpu import GpuSession
    ds = label(small_ternary(4, 48, seed=21), model, O.Oracle, 1.0, 0.1)
    pert = Model(model.family, model.ntypes,
                 [Table(t.kind, t.values * 1.02, t.rmin, t.rmax, t.form) for t in model.tables])
    g = GpuSession(0, precision)
    g.upload(ds)
    g.set_model(pert)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(pert)
    return g, o


def _close(a, b, tol, what):
    err = np.max(np.abs(np.asarray(a) - np.asarray(b)) / (1.0 + np.abs(b)))
    assert err <= tol, f"{what}: {err:.3e}"


@pytest.mark.parametrize("name", list(MODELS))
def test_residual_fp64(name):
    g, o = _sessions(MODELS[name](), "fp64")
    a, b = g.eval(1.0, 0.1), o.eval(1.0, 0.1)
    for k in ("forces", "energy", "stress", "F", "limit"):
        _close(a[k], b[k], 1e-9, k)
    assert abs(a["obj"] - b["obj"]) <= 1e-9 * abs(b["obj"])


@pytest.mark.parametrize("name", list(MODELS))
def test_residual_fp32(name):
    g, o = _sessions(MODELS[name](), "fp32")
    a, b = g.eval(1.0, 0.1), o.eval(1.0, 0.1)
    assert np.max(np.abs(a["forces"] - b["forces"])) <= 2e-5 * np.max(np.abs(b["forces"]))
    assert abs(a["obj"] - b["obj"]) <= 1e-4 * abs(b["obj"])


@pytest.mark.parametrize("name", list(MODELS))
def test_jacobian_fp64_central_differences(name):
    g, o = _sessions(MODELS[name](), "fp64")
    J = g.jacobian(1.0, 0.1)["J"]
    Jo = o.jacobian_analytic(1.0, 0.1)
    scale = np.max(np.abs(Jo), axis=0)
    assert np.all(np.abs(J - Jo) <= 1e-5 * scale[None, :] + 1e-8)


def test_jacobian_fp32_refused():
    g, _ = _sessions(pair_model(), "fp32")
    with pytest.raises(FsError) as e:
        g.jacobian(1.0, 0.1)
    assert e.value.code == FS_ERR_UNSUPPORTED
