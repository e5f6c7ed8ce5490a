"""The data formats on either side of the path (forcesmith_b200/io.py) and
the evaluate report (forcesmith_b200/evaluate.py), on CPU with the oracle."""
import json
import math
import os

import numpy as np
import pytest

from forcesmith_b200 import io, synth
from forcesmith_b200.abi import FS_FAMILY_EAM, FS_FAMILY_PAIR, FS_TABLE_ANALYTIC, Model, Table
from forcesmith_b200.evaluate import evaluate_report
from oracle import api as O
from tests.helpers import label, small_ternary, ternary_models


def test_species_slots_by_atomic_number():
    assert io.species_slots(["Zr", "Cu", "Al", "Cu"]) == ["Al", "Cu", "Zr"]
    with pytest.raises(io.FormatError):
        io.species_slots(["Xx"])


def test_config_stress_order_and_box_columns():
    txt = json.dumps([{"name": "c0", "X": [3, 0, 0], "Y": [1, 4, 0], "Z": [0, 0.5, 5], "E": -1.5, "W": 2.0,
                       "S": [1, 2, 3, 4, 5, 6],
                       "atoms": [{"element": "Cu", "position": [0, 0, 0], "force": [1, 2, 3]},
                                 {"element": "Al", "position": [1, 1, 1]}]}])
    ds, slots, names, w = io.read_configs(txt)
    assert slots == ["Al", "Cu"] and names == ["c0"] and w[0] == 2.0
    assert list(ds.type) == [1, 0]
    B = ds.box9[0].reshape(3, 3)
    np.testing.assert_array_equal(B[:, 0], [3, 0, 0])
    np.testing.assert_array_equal(B[:, 1], [1, 4, 0])
    S = ds.ref_stress9[0].reshape(3, 3)
    # S = xx, yy, zz, xy, yz, xz (config_reader.cpp:78-91)
    assert (S[0, 0], S[1, 1], S[2, 2], S[0, 1], S[1, 2], S[0, 2]) == (1, 2, 3, 4, 5, 6)
    assert np.allclose(S, S.T)
    np.testing.assert_array_equal(ds.ref_force[1], [0, 0, 0])


def test_config_roundtrip():
    ds = label(small_ternary(3, 20, seed=4), ternary_models(20)[0], O.Oracle, 1.0, 0.1)
    slots = ["Al", "Cu", "Zr"]
    back, s2, names, w = io.read_configs(io.write_configs(ds, slots, names=["a", "b", "c"]))
    assert s2 == slots and names == ["a", "b", "c"]
    for k in ("natoms", "box9", "pos", "type", "ref_force", "ref_energy"):
        np.testing.assert_array_equal(getattr(back, k), getattr(ds, k))
    # the format stores six stress components: the upper triangle (the
    # residual's Voigt rows 00, 11, 22, 01, 02, 12) survives exactly
    iu = np.triu_indices(3)
    for c in range(ds.n_cfg):
        np.testing.assert_array_equal(back.ref_stress9[c].reshape(3, 3)[iu], ds.ref_stress9[c].reshape(3, 3)[iu])


def _tables_equal(a, b):
    assert a.family == b.family and a.ntypes == b.ntypes and len(a.tables) == len(b.tables)
    for s, t in zip(a.tables, b.tables):
        assert s.kind == t.kind and s.form == t.form and s.rmin == t.rmin and s.rmax == t.rmax
        np.testing.assert_array_equal(s.values, t.values)


def test_model_roundtrip():
    _, spl = ternary_models(20)
    _tables_equal(io.read_model(io.write_model(spl)), spl)
    pair = Model(FS_FAMILY_PAIR, 2, [Table.analytic("lj", [0.2, 2.5], 0.5, 6.0),
                                     Table.analytic("morse", [0.3, 1.5, 2.8], 0.5, 6.0,
                                                    lower=[0.1, 1.0, 2.0], upper=[1.0, 3.0, 3.5]),
                                     Table.analytic("born", [0.5, 0.35, 2.0, 8.0, 6.0], 0.5, 6.0,
                                                    fixed=[0, 1, 0, 0, 1])])
    back = io.read_model(io.write_model(pair))
    _tables_equal(back, pair)
    np.testing.assert_array_equal(back.tables[1].lower, [0.1, 1.0, 2.0])
    np.testing.assert_array_equal(back.tables[2].fixed, [0, 1, 0, 0, 1])


def test_tersoff_and_angular_models():
    """tersoff: one parameter block per pair slot, ω free only when given
    (force_model_reader.cpp:166-196); angular: pair, radial, angular sections."""
    from forcesmith_b200.abi import FS_FAMILY_ANGULAR, FS_FAMILY_TERSOFF
    blk = dict(A=1830.8, B=471.18, **{"lambda": 2.4799}, mu=1.7322, beta=1.1e-6, n=0.78734,
               c=1.0039e5, d=16.217, h=-0.59825, R={"value": 2.7, "min": 2.5, "max": 2.9}, S=3.0)
    m = io.read_model(json.dumps({"model": "tersoff", "ntypes": 2,
                                  "potentials": [blk, dict(blk, omega=0.9), blk]}))
    assert m.family == FS_FAMILY_TERSOFF and len(m.tables) == 3
    assert m.tables[0].fixed[11] == 1 and m.tables[0].values[11] == 1.0
    assert m.tables[1].fixed[11] == 0 and m.tables[1].values[11] == 0.9
    assert m.tables[0].lower[9] == 2.5 and m.tables[0].values[2] == 2.4799
    _tables_equal(io.read_model(io.write_model(m)), m)
    with pytest.raises(io.FormatError):
        io.read_model(json.dumps({"model": "tersoff", "ntypes": 1, "potentials": [dict(blk, A=None) | {"A": 1.0}] * 2}))
    ang = Model(FS_FAMILY_ANGULAR, 1, [Table.analytic("lj", [1.0, 1.0], 0.1, 20.0),
                                       Table.spline(0.0, 5.0, [1.0, 0.6, 0.3, 0.1, 0.0]),
                                       Table.analytic("harmonic", [1.0, -0.5], -1.0, 1.0)])
    back = io.read_model(io.write_model(ang))
    assert back.family == FS_FAMILY_ANGULAR
    _tables_equal(back, ang)


def test_ml_acsf_model():
    """build_ml / parse_linear_head (force_model_reader.cpp:217-333)."""
    from forcesmith_b200.abi import FS_FAMILY_ACSF, acsf_size
    j = {"model": "ml", "ntypes": 2,
         "descriptor": {"type": "symmetry_functions", "rcut": 5.0, "g1": 1, "g2": [{"eta": 0.5, "rs": 1.0}, {"eta": 1.0}],
                        "g4": [{"eta": 0.1, "zeta": 2.0, "lambda": -1.0}]},
         "heads": [{"type": "linear", "coeffs": [0.1] * 9, "bias": -3.0},
                   {"coeffs": [0.2] * 9, "bias": -2.0, "bias_fixed": False, "fixed": True}]}
    m = io.read_model(json.dumps(j))
    assert m.family == FS_FAMILY_ACSF and acsf_size(m.tables[0], 2) == 9
    assert m.tables[0].values[0] == 5.0 and list(m.tables[0].values[1:6]) == [1, 2, 0, 1, 0]
    assert m.tables[1].fixed[-1] == 1 and m.tables[2].fixed[-1] == 0 and np.all(m.tables[2].fixed[:-1] == 1)
    _tables_equal(io.read_model(io.write_model(m)), m)
    with pytest.raises(io.FormatError):
        io.read_model(json.dumps(dict(j, heads=j["heads"][:1])))
    with pytest.raises(io.FormatError):
        io.read_model(json.dumps(dict(j, descriptor={"type": "soap"})))


def test_model_json_forms_and_errors():
    eam = {"model": "eam", "ntypes": 1,
           "pair": {"format": "analytic", "potentials": [{"type": "buck", "rmin": 0.5, "rmax": 6.0, "A": 900.0,
                                                           "rho": {"value": 0.3, "min": 0.1, "max": 1.0},
                                                           "C": {"value": 10.0, "fixed": True}}]},
           "density": {"format": "analytic", "potentials": [{"type": "exp", "rmin": 0.5, "rmax": 6.0,
                                                              "A": 4.0, "B": 1.2}]},
           "embedding": {"format": "tabulated", "potentials": [{"rmin": 0, "rmax": 30, "knots": [0, -1, -1.4, -1.7],
                                                                "fixed": True}]}}
    m = io.read_model(json.dumps(eam))
    assert m.family == FS_FAMILY_EAM and len(m.tables) == 3
    assert m.tables[0].kind == FS_TABLE_ANALYTIC and m.tables[0].lower[1] == 0.1 and m.tables[0].fixed[2] == 1
    assert np.all(m.tables[2].fixed == 1)
    bare = {"format": "tabulated", "potentials": [{"rmin": 1, "rmax": 5, "knots": [1, 0.5, 0]}] * 3}
    assert io.read_model(json.dumps(bare)).ntypes == 2
    with pytest.raises(io.FormatError):
        io.read_model(json.dumps({"format": "tabulated", "potentials": [bare["potentials"][0]] * 2}))
    bad = dict(eam, pair={"format": "analytic", "potentials": [{"type": "nope", "rmin": 0, "rmax": 1}]})
    with pytest.raises(io.FormatError):
        io.read_model(json.dumps(bad))
    # a global without links is still a free parameter, after the tables'
    g = io.read_model(json.dumps(dict(eam, globals={"g": {"value": 1.5}})))
    assert g.free_values()[-1] == 1.5 and g.free_values().size == m.free_values().size + 1


def test_evaluate_report_sums_to_objective():
    true, start = ternary_models(20)
    ds = label(small_ternary(3, 24, seed=8), true, O.Oracle, 1.0, 0.1)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(start)
    rep = evaluate_report(o, ds, 1.0, 0.1, names=["x", "y", "z"])
    obj = o.eval(1.0, 0.1, want=("obj",))["obj"]
    assert rep["nconf"] == 3 and rep["configs"][1]["name"] == "y"
    assert rep["total_sumsq"] == pytest.approx(obj, rel=1e-12)
    assert sum(c["sumsq"] for c in rep["configs"]) == pytest.approx(rep["total_sumsq"], rel=1e-14)
    assert len(rep["configs"][0]["atoms"]) == 24 and len(rep["configs"][0]["calc_stress"]) == 6


# the reference's data/Al99.eam.alloy: FORCESMITH_SRC names the Forcesmith
# source tree (the test is skipped without it)
SETFL = os.path.join(os.environ.get("FORCESMITH_SRC", "/nonexistent"), "data", "Al99.eam.alloy")


@pytest.mark.skipif(not os.path.exists(SETFL), reason="FORCESMITH_SRC does not name the Forcesmith sources")
def test_read_setfl_matches_fixture_pin():
    model, hdr = io.read_setfl(SETFL)
    assert hdr["element"] == "Al" and hdr["nr"] == 10000 and math.isclose(hdr["rc"], 6.28721)
    ideal = synth.fcc(1, 3, 4.05, 0.0, 1.0, 1.0, seed=1)
    o = O.Oracle()
    o.upload(ideal.with_labels(np.zeros((ideal.n_atoms, 3)), np.zeros(1), np.zeros((1, 9))))
    o.set_model(model)
    e = o.eval(1.0, 0.0, want=("energy",))["energy"][0] / ideal.n_atoms
    assert abs(e + 3.36) < 1e-5


def test_ml_standardization_round_trip():
    """finish_ml / add_standardization (force_model_reader.cpp:261-281,
    output_writer.cpp:155-168): one {mean, inv_std} per species; an empty
    entry (a species without training atoms) reads as the identity."""
    from forcesmith_b200.abi import FS_TABLE_STANDARDIZATION
    j = {"model": "ml", "ntypes": 2,
         "descriptor": {"type": "acsf", "rcut": 5.0, "g2": [{"eta": 0.5, "rs": 1.0}]},
         "heads": [{"coeffs": [0.1, 0.2], "bias": -3.0}, {"coeffs": [0.3, 0.4], "bias": -2.0}],
         "standardization": [{"mean": [0.5, 0.25], "inv_std": [2.0, 0.0]}, {"mean": [], "inv_std": []}]}
    m = io.read_model(json.dumps(j))
    assert len(m.tables) == 5 and m.tables[3].kind == FS_TABLE_STANDARDIZATION
    assert m.tables[3].values.tolist() == [0.5, 0.25, 2.0, 0.0] and m.tables[4].values.tolist() == [0, 0, 1, 1]
    assert np.all(m.tables[3].fixed == 1)
    back = io.read_model(io.write_model(m))
    _tables_equal(back, m)
    with pytest.raises(io.FormatError):
        io.read_model(json.dumps(dict(j, standardization=j["standardization"][:1])))
