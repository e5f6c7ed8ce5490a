"""fs_gpu_tabulate (the writers' sampler on the device) and global
parameters on the device, against the oracle.

  tabulate   value and d/dr of spline and analytic tables at the current
             parameters, FP64 whatever the context precision:
             |v − v_oracle| ≤ 1e-12·(1 + |v|), the same for d/dr; the native
             JSON, LAMMPS and IMD texts written from the device sampler
             match the ones written from the oracle's (knots 1e-12; the
             6-digit texts to their last digit)
  globals    the EAM model with one smooth-cutoff h shared by a morse_sc pair
             and an exp_decay_sc density: parameter count, gather order and
             bounds as the oracle's; set_params broadcasts h (forces, energy,
             stress, limit 1e-9·(1 + |x|) against the oracle at a moved h);
             with h free the Jacobian is the reference's central differences
             (the oracle's, 1e-7·(1 + |J|)); with h fixed the analytic one
"""
import json

import numpy as np
import pytest

from forcesmith_b200 import io
from forcesmith_b200.abi import Table
from oracle import api as O
from tests.helpers import small_ternary, with_zero_labels
from tests.test_io_reference_cases_cpu import EAM_GLOBAL_H, oracle_sampler, oracle_vd, pair_model

pytestmark = pytest.mark.gpu


def _session(model, precision="fp64", ds=None):
    from forcesmith_b200.gpu import GpuSession
    g = GpuSession(0, precision)
    if ds is not None:
        g.upload(ds)
    g.set_model(model, prepare=ds is not None)
    return g


def _models():
    eam = io.read_model(json.dumps(EAM_GLOBAL_H))
    spline = io.read_model(json.dumps({
        "model": "eam", "ntypes": 1,
        "pair": {"format": "tabulated", "potentials": [{"rmin": 1.5, "rmax": 6.0,
                                                        "knots": [2.0, 1.0, 0.1, -0.2, -0.1, 0.0]}]},
        "density": {"format": "tabulated", "potentials": [{"rmin": 1.5, "rmax": 6.0,
                                                           "knots": [1.0, 0.6, 0.3, 0.1, 0.02, 0.0]}]},
        "embedding": {"format": "tabulated", "potentials": [{"rmin": 0.0, "rmax": 4.0,
                                                             "knots": [0.0, -1.0, -1.4, -1.6, -1.7]}]}}))
    return {"analytic_globals": eam, "spline": spline, "pair": pair_model()}


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", ["analytic_globals", "spline", "pair"])
def test_tabulate_matches_oracle(name, precision):
    m = _models()[name]
    g = _session(m, precision)
    for k, t in enumerate(m.tables):
        r = np.linspace(t.rmin - 0.3, t.rmax + 0.3, 301)  # the linear extension of a spline too
        if t.kind != 0:
            r = np.linspace(max(t.rmin, 1e-3), t.rmax, 301)
        v, d = g.tabulate(k, r)
        ref = np.array([oracle_vd(t, q) for q in r])
        assert np.all(np.abs(v - ref[:, 0]) <= 1e-12 * (1 + np.abs(ref[:, 0]))), (k, np.max(np.abs(v - ref[:, 0])))
        assert np.all(np.abs(d - ref[:, 1]) <= 1e-12 * (1 + np.abs(ref[:, 1]))), (k, np.max(np.abs(d - ref[:, 1])))


def test_tabulate_follows_set_params_and_writers_agree():
    m = _models()["pair"]
    g = _session(m)
    x = m.free_values() * 1.03
    g.set_params(x)
    m2 = m.with_values(x)
    dev, ora = io.session_sampler(g), oracle_sampler(m2)
    a, b = json.loads(io.write_native(m2, dev)), json.loads(io.write_native(m2, ora))
    for pa, pb in zip(a["potentials"], b["potentials"]):
        assert (pa["rmin"], pa["rmax"]) == (pb["rmin"], pb["rmax"])
        np.testing.assert_allclose(pa["knots"], pb["knots"], rtol=1e-12, atol=1e-14)
    for write in (io.write_lammps, io.write_imd):
        ta, tb = write(m2, dev).split(), write(m2, ora).split()
        assert len(ta) == len(tb)
        for u, w in zip(ta, tb):  # 6-digit text: a last digit may round either way
            try:
                assert abs(float(u) - float(w)) <= 2e-5 * max(abs(float(w)), 1e-300)
            except ValueError:
                assert u == w


def test_tabulate_rejects_non_radial_tables():
    from forcesmith_b200.abi import FS_FAMILY_SW, Model
    sw = Model(FS_FAMILY_SW, 1, [Table.sw(7.05, 0.60, 4.0, 0.0, 2.0951, 3.7712, 1.2, 3.7712),
                                 Table(3, np.array([21.0]), 0.0, 0.0, 0)])
    g = _session(sw)
    with pytest.raises(Exception, match="not a radial table"):
        g.tabulate(0, np.array([2.0]))


def _pair(model, precision="fp64"):
    ds = small_ternary(2, 24, seed=5)
    ds.type[:] = 0
    o = O.Oracle()
    o.upload(with_zero_labels(ds))
    o.set_model(model)
    lab = o.eval(1.0, 0.1)
    ds = ds.with_labels(lab["forces"] * 1.01, lab["energy"] + 0.05, lab["stress"] * 0.98)
    o.upload(ds)
    o.set_model(model)
    return _session(model, precision, ds), o


def test_globals_layout_and_broadcast():
    m = _models()["analytic_globals"]
    g, o = _pair(m)
    assert g.D == o.D == 8
    np.testing.assert_array_equal(g.gather_params(), o.gather_params())
    lo, hi = g.gather_bounds()
    olo, ohi = o.gather_bounds()
    np.testing.assert_array_equal(lo, olo)
    np.testing.assert_array_equal(hi, ohi)
    x = o.gather_params()
    x[-1] = 1.7  # the shared h
    x[0] *= 1.05
    g.set_params(x)
    o.set_params(x)
    np.testing.assert_array_equal(g.gather_params(), x)
    a, b = g.eval(1.0, 0.1), o.eval(1.0, 0.1)
    for key in ("forces", "energy", "stress", "limit", "F"):
        err = np.max(np.abs(a[key] - b[key]) / (1.0 + np.abs(b[key])))
        assert err <= 1e-9, (key, err)


def test_globals_free_jacobian_is_central_differences():
    m = _models()["analytic_globals"]
    g, o = _pair(m)
    J = g.jacobian(1.0, 0.1)["J"]
    Jf = o.jacobian_fd(1.0, 0.1)
    assert J.shape == Jf.shape
    assert np.all(np.abs(J - Jf) <= 1e-7 * (1.0 + np.abs(Jf))), np.max(np.abs(J - Jf))
    # the global's column is the sum over its two links
    assert np.max(np.abs(Jf[:, -1])) > 0.0


def test_globals_fixed_jacobian_is_analytic():
    doc = json.loads(json.dumps(EAM_GLOBAL_H))
    doc["globals"]["h"]["fixed"] = True
    m = io.read_model(json.dumps(doc))
    assert m.free_values().size == 7
    g, o = _pair(m)
    J = g.jacobian(1.0, 0.1)["J"]
    Ja = o.jacobian_analytic(1.0, 0.1)
    assert np.all(np.abs(J - Ja) <= 1e-9 * (1.0 + np.abs(Ja))), np.max(np.abs(J - Ja))
