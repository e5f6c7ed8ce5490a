"""Analytic radial tables on the device (the reference's AnalyticForm
potentials, include/forcesmith/potentials/analytic_potential.hpp), against
the oracle.

  FP64 residual   |Δ| ≤ 1e-9·(1 + |x|) (forces, energies, stress, F rows)
  FP32 residual   forces 2e-5·max|F|, objective 1e-4 relative
  Jacobian, every table analytic: the device's exact chain rule (the
                  reference's write_param_jacobian, eam_force.cpp:108-279,
                  pair_force.cpp:80-111) against the oracle's analytic
                  Jacobian: FP64 1e-9·(1 + |J|), FP32 1e-4·max|J column|;
                  and against the oracle's central differences, the
                  reference's bar 1e-5·max|column| + 1e-8
                  (test_param_jacobian.cpp:70)
  Jacobian, analytic and spline tables mixed: the reference's central
                  differences on the device (FP64 contexts), 1e-5·max|column|
                  + 1e-8 against the oracle's analytic Jacobian; FP32 refused
Every one of the 34 forms is checked as a one-species pair model: residual
and exact Jacobian in FP64 against the oracle.
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


def eam_model_b():
    """Other forms in the three EAM roles, and an embedding span that clamps
    the atoms (their density derivatives go to the limit row)."""
    pairs = [Table.analytic("double_exp", [0.6, 0.8 + 0.05 * k, 2.6, 1.5, 2.0], 0.5, RC) for k in range(3)] + \
            [Table.analytic("tersoff_mix", [2.0 + 0.2 * k, 1.6], 0.5, RC) for k in range(3)]
    dens = [Table.analytic("mishin", [1.2 + 0.1 * k, 0.3, 0.0, 1.0, 2.0, 1.1], 0.5, RC) for k in range(3)]
    emb = [Table.analytic("universal", [-0.8 - 0.1 * k, 0.5, 1.5, 0.01], 0.0, 2.5 + k) for k in range(3)]
    return Model(FS_FAMILY_EAM, 3, pairs + dens + emb)


ANALYTIC = {"pair": pair_model, "eam": eam_model, "eam_b": eam_model_b}


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", list(ANALYTIC))
def test_jacobian_exact(name, precision):
    g, o = _sessions(ANALYTIC[name](), precision)
    res = g.jacobian(1.0, 0.1)
    Ja = o.jacobian_analytic(1.0, 0.1)
    assert res["J"].shape == Ja.shape
    if precision == "fp64":
        _close(res["J"], Ja, 1e-9, "J")
        F = o.eval(1.0, 0.1)["F"]
        JtJ, Jtr = O.normal_equations(Ja, F)
        _close(res["JtJ"], JtJ, 1e-9, "JtJ")
        _close(res["Jtr"], Jtr, 1e-9, "Jtr")
        Jf = o.jacobian_fd(1.0, 0.1)
        scale = np.max(np.abs(Jf), axis=0)
        assert np.all(np.abs(res["J"] - Jf) <= 1e-5 * scale[None, :] + 1e-8)
    else:
        colmax = np.abs(Ja).max(axis=0) + 1e-30
        assert np.max(np.abs(res["J"] - Ja) / colmax) <= 1e-4


def test_eam_b_clamps_atoms():
    """The embedding spans of eam_model_b clamp the atoms' densities: the
    limit rows are live, and their Jacobian rows match the oracle's (checked
    in test_jacobian_exact)."""
    _, o = _sessions(eam_model_b(), "fp64")
    assert np.any(o.eval(1.0, 0.1)["limit"] > 0)


def test_jacobian_mixed_fp64_central_differences():
    g, o = _sessions(eam_model(True), "fp64")
    J = g.jacobian(1.0, 0.1)["J"]
    Jo = o.jacobian_analytic(1.0, 0.1)
    scale = np.max(np.abs(Jo), axis=0)
    assert np.all(np.abs(J - Jo) <= 1e-5 * scale[None, :] + 1e-8)


def test_jacobian_mixed_fp32_refused():
    g, _ = _sessions(eam_model(True), "fp32")
    with pytest.raises(FsError) as e:
        g.jacobian(1.0, 0.1)
    assert e.value.code == FS_ERR_UNSUPPORTED


def _form_cases():
    from tests.test_oracle_forms_cpu import reference_values
    return [(name, p) for name, p, _ in reference_values(2.0)]


@pytest.mark.parametrize("name,params", _form_cases(), ids=[c[0] for c in _form_cases()])
def test_every_form_residual_and_jacobian_fp64(name, params):
    """One species, one pair table of the form (the parameters of the
    reference's formula test), gate [0.5, 5.5]: residual and exact Jacobian
    against the oracle."""
    from forcesmith_b200.gpu import GpuSession
    model = Model(FS_FAMILY_PAIR, 1, [Table.analytic(name, params, 0.5, RC)])
    ds = small_ternary(3, 40, seed=23)
    ds.type[:] = 0
    ds = label(ds, Model(FS_FAMILY_PAIR, 1, [Table.analytic(name, np.asarray(params) * 1.01, 0.5, RC)]),
               O.Oracle, 1.0, 0.1)
    g = GpuSession(0, "fp64")
    g.upload(ds)
    g.set_model(model)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model)
    a, b = g.eval(1.0, 0.1), o.eval(1.0, 0.1)
    for k in ("forces", "energy", "stress", "F"):
        _close(a[k], b[k], 1e-9, f"{name} {k}")
    J = g.jacobian(1.0, 0.1)["J"]
    _close(J, o.jacobian_analytic(1.0, 0.1), 1e-9, f"{name} J")
