"""Parity of the benchmark workloads at their full sizes, FP32 device path
against the FP64 oracle (the reference's CPU arithmetic).

Workloads (seeded, the shapes the benchmark times):
  ternary EAM   500 configurations × 256 atoms, 6 φ + 3 ρ + 3 F splines of
                20 knots (D = 240), w_e = 1, w_s = 0.1 (388,000 rows)
  SW Si         1000 diamond configurations of 64, 216 or 512 atoms, 7 free
                Stillinger–Weber parameters, w_e = 1, w_s = 0.1
  DE population the ternary model on 200 configurations of 32–512 atoms,
                20 trial vectors

Force bar (north star: forces within 1e-5 relative of the FP64 oracle),
stated per component and as a norm:
  per component  |F_ia − F_ia^ref| ≤ 1e-5 · (|F_i^ref| + 1 eV/Å)
                 (|F_i^ref| the atom's force magnitude; the 1 eV/Å floor
                 stands for the size of the pair terms an atom's force sums,
                 which sets FP32's rounding for atoms whose net force nearly
                 cancels)
  norm           ‖F − F^ref‖₂ ≤ 1e-5 · ‖F^ref‖₂ over every component
Other bars: energies 1e-6 relative, stress 1e-5 of the largest stress
component, objective 1e-5 relative, Jᵀr 1e-5 of its largest entry, JᵀJ 1e-4
of √(JᵀJ_aa·JᵀJ_bb) (3×TF32 products of an FP32 Jacobian), population
objectives 1e-5 relative.  The FP64 device path is held to 1e-9·(1 + |x|).
Each test prints the errors it measured (pytest -s shows them).

Measured on a B200 (FP32 device path against the FP64 oracle):
  ternary  forces per component 2.9e-6 (1.4e-5 without the floor), norm
           1.4e-7, max 1.4e-5 eV/Å; energies 2.9e-8; stress 7.5e-8;
           objective 2.0e-7; Jᵀr 1.9e-7; JᵀJ 3.0e-5
  SW       forces per component 2.8e-6, norm 4.0e-7; energies 4.4e-8;
           objective 2.9e-8; Jᵀr against central differences 1.3e-8
  DE       population objectives 1.6e-6
"""
import json

import numpy as np
import pytest

from forcesmith_b200 import synth
from oracle import api as O

pytestmark = pytest.mark.gpu


def _gpu(precision):
    from forcesmith_b200.gpu import GpuSession
    return GpuSession(0, precision)


def _labelled(ds, true, start, w_e, w_s):
    """Labels from `true` in FP64 (oracle); returns the dataset and an oracle
    session at `start`."""
    o = O.Oracle()
    o.upload(ds)
    o.set_model(true)
    lab = o.eval(w_e, w_s)
    ds = ds.with_labels(lab["forces"], lab["energy"], lab["stress"])
    o.set_references(ds)
    o.set_model(start)
    return ds, o


def force_errors(f, ref):
    f = np.asarray(f, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    mag = np.linalg.norm(ref, axis=1, keepdims=True)
    d = np.abs(f - ref)
    return {"per_component": float(np.max(d / (mag + 1.0))),
            "per_component_no_floor": float(np.max(d / np.maximum(mag, 1e-300))),
            "norm": float(np.linalg.norm(f - ref) / np.linalg.norm(ref)),
            "max_abs_eV_per_A": float(d.max())}


def _report(name, errs):
    print(f"\n{name}: " + json.dumps({k: float(f"{v:.3e}") for k, v in errs.items()}))


@pytest.fixture(scope="module")
def ternary():
    O.set_threads(0)
    true = synth.ternary_true_model(20)
    start = synth.perturb(true, 0.95, 1.05, seed=7)
    ds, o = _labelled(synth.ternary_geometry(), true, start, 1.0, 0.1)
    ref = o.eval(1.0, 0.1)
    return ds, start, o, ref


def test_ternary_fp32_residual_full_size(ternary):
    ds, start, _, ro = ternary
    g = _gpu("fp32")
    g.upload(ds)
    g.set_model(start)
    rg = g.eval(1.0, 0.1)
    g.close()
    e = force_errors(rg["forces"], ro["forces"])
    e["energy_rel"] = float(np.max(np.abs(rg["energy"] - ro["energy"]) / np.abs(ro["energy"])))
    e["stress"] = float(np.max(np.abs(rg["stress"] - ro["stress"])) / np.max(np.abs(ro["stress"])))
    e["objective_rel"] = abs(rg["obj"] - ro["obj"]) / ro["obj"]
    _report("ternary FP32 residual vs FP64 oracle (500 x 256)", e)
    assert e["per_component"] <= 1e-5
    assert e["norm"] <= 1e-5
    assert e["energy_rel"] <= 1e-6
    assert e["stress"] <= 1e-5
    assert e["objective_rel"] <= 1e-5


def test_ternary_fp32_normal_equations_full_size(ternary):
    ds, start, o, ro = ternary
    g = _gpu("fp32")
    g.upload(ds)
    g.set_model(start)
    res = g.jacobian(1.0, 0.1, want_J=False)
    g.close()
    J = o.jacobian_analytic(1.0, 0.1)
    JtJ, Jtr = J.T @ J, J.T @ ro["F"]
    del J
    d = np.sqrt(np.outer(np.diag(JtJ), np.diag(JtJ))) + 1e-300
    e = {"JtJ": float(np.max(np.abs(res["JtJ"] - JtJ) / d)),
         "Jtr": float(np.max(np.abs(res["Jtr"] - Jtr)) / np.max(np.abs(Jtr))),
         "objective_rel": abs(res["obj"] - ro["obj"]) / ro["obj"]}
    _report("ternary FP32 JtJ / Jtr vs FP64 analytic oracle (500 x 256)", e)
    assert e["JtJ"] <= 1e-4
    assert e["Jtr"] <= 1e-5
    assert e["objective_rel"] <= 1e-5


def test_ternary_fp64_full_size(ternary):
    ds, start, _, ro = ternary
    g = _gpu("fp64")
    g.upload(ds)
    g.set_model(start)
    rg = g.eval(1.0, 0.1)
    g.close()
    for k in ("forces", "energy", "stress", "F"):
        err = float(np.max(np.abs(rg[k] - ro[k]) / (1.0 + np.abs(ro[k]))))
        assert err <= 1e-9, (k, err)
    assert abs(rg["obj"] - ro["obj"]) <= 1e-9 * ro["obj"]


def test_sw_fp32_full_size():
    O.set_threads(0)
    ds, o = _labelled(synth.diamond(1000), synth.sw_model(), synth.sw_start_model(), 1.0, 0.1)
    ro = o.eval(1.0, 0.1)
    g = _gpu("fp32")
    g.upload(ds)
    g.set_model(synth.sw_start_model())
    rg = g.eval(1.0, 0.1)
    res = g.jacobian(1.0, 0.1, want_J=False)
    g.close()
    e = force_errors(rg["forces"], ro["forces"])
    e["energy_rel"] = float(np.max(np.abs(rg["energy"] - ro["energy"]) / np.abs(ro["energy"])))
    e["stress"] = float(np.max(np.abs(rg["stress"] - ro["stress"])) / np.max(np.abs(ro["stress"])))
    e["objective_rel"] = abs(rg["obj"] - ro["obj"]) / ro["obj"]
    # the reference's own Jacobian for SW: central differences (h = 1e-5)
    Jf = o.jacobian_fd(1.0, 0.1)
    Jtr = Jf.T @ ro["F"]
    e["Jtr_vs_central_differences"] = float(np.max(np.abs(res["Jtr"] - Jtr)) / np.max(np.abs(Jtr)))
    _report("SW FP32 vs FP64 oracle (1000 configs)", e)
    assert e["per_component"] <= 1e-5
    assert e["norm"] <= 1e-5
    assert e["energy_rel"] <= 1e-6
    assert e["stress"] <= 1e-5
    assert e["objective_rel"] <= 1e-5
    assert e["Jtr_vs_central_differences"] <= 1e-4


def test_population_fp32_de_workload():
    O.set_threads(0)
    true = synth.ternary_true_model(20)
    start = synth.perturb(true, 0.95, 1.05, seed=7)
    ds, o = _labelled(synth.de_geometry(), true, start, 1.0, 0.0)
    g = _gpu("fp32")
    g.upload(ds)
    g.set_model(start)
    x0 = g.gather_params()
    xs = np.stack([x0 * synth.uniform(x0.size, 0.97, 1.03, 300 + k) for k in range(20)])
    og = g.eval_population(xs, 1.0, 0.0)
    g.close()
    oo = o.eval_population(xs, 1.0, 0.0)
    err = float(np.max(np.abs(og - oo) / oo))
    _report("DE population FP32 vs FP64 oracle (200 configs, 20 trials)", {"objective_rel": err})
    assert err <= 1e-5
