"""Tersoff on the device against the oracle (through the C ABI).

Tolerances:
  FP64  forces, energy, stress, F rows   |Δ| ≤ 1e-9·(1 + |x|); objective 1e-9 relative
  FP32  forces                           |Δ| ≤ 2e-5·max|F|;    objective 1e-4 relative
  Jacobian (FP64 central differences, h = 1e-5, the reference's method for
  Tersoff, against the oracle's own central differences)
                                         |ΔJ| ≤ 1e-5·max|J column| + 1e-7
    (both sides difference FP64 residuals summed in different orders: for the
    energy rows that noise is ~1e-11 of |E| ≈ 760, divided by 2h = 2e-5; a
    wrong parameter order or cutoff rebuild would be off by O(1))
"""
import numpy as np
import pytest

from forcesmith_b200 import synth
from forcesmith_b200.abi import FS_FAMILY_TERSOFF, Model, Table
from oracle import api as O
from tests.helpers import label
from tests.test_oracle_tersoff_cpu import SI

pytestmark = pytest.mark.gpu


def si_model(scale=1.0, nt=1):
    tabs = []
    for s in range(nt * (nt + 1) // 2):
        f = 1.0 + 0.03 * s
        p = dict(SI, A=SI["A"] * scale * f, B=SI["B"] * (2.0 - f), lam=SI["lam"] * f, R=SI["R"] - 0.05 * s)
        tabs.append(Table.tersoff(**p))
    return Model(FS_FAMILY_TERSOFF, nt, tabs)


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


@pytest.fixture(scope="module", params=[1, 2], ids=["si", "binary"])
def case(request):
    nt = request.param
    ds = synth.diamond(4, cells=(2, 3), seed=53)
    if nt == 2:
        ds.type[:] = np.random.default_rng(3).integers(0, 2, ds.type.size)
    true = si_model(1.0, nt)
    ds = label(ds, true, O.Oracle, 1.0, 0.2)
    return ds, si_model(1.04, nt)


def test_tersoff_residual_fp64(case):
    ds, start = case
    g, o = _pair(ds, start, "fp64")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    _close(rg["forces"], ro["forces"], 1e-9, "forces")
    _close(rg["energy"], ro["energy"], 1e-9, "energy")
    _close(rg["stress"], ro["stress"], 1e-9, "stress")
    _close(rg["F"], ro["F"], 1e-9, "F")
    assert abs(rg["obj"] - ro["obj"]) <= 1e-9 * ro["obj"]


def test_tersoff_residual_fp32(case):
    ds, start = case
    g, o = _pair(ds, start, "fp32")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    assert np.max(np.abs(rg["forces"] - ro["forces"])) <= 2e-5 * np.max(np.abs(ro["forces"]))
    assert abs(rg["obj"] - ro["obj"]) <= 1e-4 * ro["obj"]


def test_tersoff_jacobian_central_differences(case):
    ds, start = case
    g, o = _pair(ds, start, "fp64")
    res = g.jacobian(1.0, 0.2)
    Jf = o.jacobian_fd(1.0, 0.2)
    assert res["J"].shape == Jf.shape and Jf.shape[1] == 11 * len(start.tables)
    # β − h < 0 for the Si β = 1.1e-6 with the reference's absolute step
    # h = 1e-5: (βζ)^n is NaN there, on the device as in the reference
    ok = np.isfinite(Jf)
    assert np.array_equal(np.isfinite(res["J"]), ok)
    colmax = np.nanmax(np.abs(Jf), axis=0)
    bar = 1e-5 * np.broadcast_to(colmax, Jf.shape) + 1e-7
    ratio = np.where(ok, np.abs(res["J"] - Jf) / bar, 0.0)
    r, c = np.unravel_index(np.argmax(ratio), ratio.shape)
    assert ratio.max() <= 1.0, (ratio.max(), r, c, res["J"][r, c], Jf[r, c], np.argwhere(ratio > 1.0)[:10].tolist())
    F = o.eval(1.0, 0.2)["F"]
    good = ok.all(axis=0)
    JtJ, Jtr = O.normal_equations(Jf[:, good], F)
    d = np.max(np.abs(res["Jtr"][good] - Jtr))
    assert d <= 1e-5 * np.max(np.abs(Jtr)), (d, np.max(np.abs(Jtr)))


def test_tersoff_fp32_jacobian_refused():
    ds = synth.diamond(2, cells=(2,), seed=5)
    from forcesmith_b200.gpu import GpuSession
    g = GpuSession(0, "fp32")
    g.upload(ds)
    g.set_model(si_model())
    with pytest.raises(RuntimeError):
        g.jacobian(1.0, 0.0)
