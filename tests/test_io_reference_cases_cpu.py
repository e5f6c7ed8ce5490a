"""The reference's reader and writer unit tests, case by case, against
forcesmith_b200.io (and the oracle where a case evaluates a potential).

  tests/unit/test_config_reader.cpp       13 cases (ConfigReader.*)
  tests/unit/test_potential_reader.cpp     8 cases (PotentialReader.*)
  tests/unit/test_force_model_reader.cpp  16 cases (ForceModelReader.*,
                                          WriteModel.*)

Each test names the reference case it restates; the inputs are the same
documents, built here as Python objects, and the assertions are the same
facts.  Where a reference case evaluates a potential (eval / deriv at a
point), the oracle evaluates the parsed table.
"""
import json
import math

import numpy as np
import pytest

from forcesmith_b200 import io
from forcesmith_b200.abi import (FS_FAMILY_ACSF, FS_FAMILY_ANGULAR, FS_FAMILY_EAM, FS_FAMILY_PAIR, FS_FAMILY_SW,
                                 FS_FAMILY_TERSOFF, FS_TABLE_SPLINE, TERSOFF_FIELDS)
from oracle import api as O


def cube(a):
    return {"X": [a, 0.0, 0.0], "Y": [0.0, a, 0.0], "Z": [0.0, 0.0, a]}


def cfg(a, E, atoms, **kw):
    return {**cube(a), "E": E, "atoms": atoms, **kw}


def atom(el, pos, force=None):
    d = {"element": el, "position": list(pos)}
    if force is not None:
        d["force"] = list(force)
    return d


def read(doc):
    return io.read_configs(doc if isinstance(doc, str) else json.dumps(doc))


# ---------------------------------------------------------------------------
# ConfigReader (test_config_reader.cpp)

def test_config_single_atom_no_forces():  # SingleAtomNoForces
    ds, slots, _, w = read([cfg(4.0, -1.5, [atom("Cu", (1.0, 2.0, 3.0))], W=2.0)])
    assert ds.n_cfg == 1 and ds.natoms[0] == 1
    assert ds.ref_energy[0] == -1.5 and w[0] == 2.0
    assert ds.type[0] == 0 and slots == ["Cu"]
    assert list(ds.pos[0]) == [1.0, 2.0, 3.0]
    assert np.linalg.norm(ds.ref_force[0]) == 0.0


def test_config_two_atoms_with_forces():  # TwoAtomsWithForces
    ds, slots, _, _ = read([cfg(5.0, -3.14, [atom("Cu", (0, 0, 0), (0.1, 0.2, 0.3)),
                                             atom("Fe", (2.5, 2.5, 2.5), (-0.1, -0.2, -0.3))])])
    assert ds.natoms[0] == 2 and ds.ref_energy[0] == -3.14
    assert slots == ["Fe", "Cu"]  # Z-sorted: Fe(26) → 0, Cu(29) → 1
    assert ds.type[0] == 1 and ds.type[1] == 0
    assert abs(ds.ref_force[0, 0] - 0.1) <= 1e-12 and abs(ds.ref_force[0, 2] - 0.3) <= 1e-12
    assert ds.pos[1, 0] == 2.5 and abs(ds.ref_force[1, 0] + 0.1) <= 1e-12


def test_config_box_vectors_stored():  # BoxVectorsStored
    doc = [{"X": [3.0, 0.1, 0.0], "Y": [0.0, 4.0, 0.2], "Z": [0.0, 0.0, 5.0], "E": 0.0,
            "atoms": [atom("Cu", (0, 0, 0))]}]
    ds, _, _, _ = read(doc)
    box = ds.box9[0].reshape(3, 3)  # columns are the lattice vectors
    assert box[0, 0] == 3.0 and box[1, 0] == 0.1 and box[2, 0] == 0.0
    assert box[0, 1] == 0.0 and box[1, 1] == 4.0 and box[2, 1] == 0.2
    assert box[2, 2] == 5.0


def test_config_stress_tensor_stored():  # StressTensorStored
    ds, _, _, _ = read([cfg(4.0, 0.0, [atom("Cu", (0, 0, 0))], S=[1.1, 2.2, 3.3, 4.4, 5.5, 6.6])])
    s = ds.ref_stress9[0].reshape(3, 3)
    assert (s[0, 0], s[1, 1], s[2, 2]) == (1.1, 2.2, 3.3)
    assert s[0, 1] == 4.4 and s[1, 0] == 4.4 and s[1, 2] == 5.5 and s[0, 2] == 6.6


def test_config_multiple_configurations():  # MultipleConfigurations
    ds, _, _, _ = read([cfg(4.0, -1.0, [atom("Cu", (0, 0, 0))]),
                        cfg(5.0, -2.0, [atom("Cu", (0, 0, 0)), atom("Fe", (2.5, 2.5, 2.5))])])
    assert ds.n_cfg == 2 and list(ds.natoms) == [1, 2]
    assert list(ds.ref_energy) == [-1.0, -2.0]


def test_config_element_type_mapping():  # ElementTypeMapping
    ds, _, _, _ = read([cfg(4.0, 0.0, [atom("Cu", (0, 0, 0))]),
                        cfg(4.0, 0.0, [atom("Fe", (1, 0, 0)), atom("Cu", (2, 0, 0))])])
    assert list(ds.type) == [1, 0, 1]  # Cu → 1, Fe → 0, across configurations


def test_config_default_weight_is_one():  # DefaultWeightIsOne
    _, _, _, w = read([cfg(4.0, 0.0, [atom("Cu", (0, 0, 0))])])
    assert w[0] == 1.0


def test_config_empty_input_returns_no_configs():  # EmptyInputReturnsNoConfigs
    ds, _, _, _ = read("[]")
    assert ds.n_cfg == 0


def test_config_minified_json_parsed():  # MinifiedJsonParsed
    text = '[{"X":[4,0,0],"Y":[0,4,0],"Z":[0,0,4],"E":-1.0,"atoms":[{"element":"Cu","position":[0,0,0]}]}]'
    ds, _, _, _ = read(text)
    assert ds.n_cfg == 1 and ds.ref_energy[0] == -1.0


@pytest.mark.parametrize("doc", [
    {"X": [4, 0, 0]},                                                   # ErrorTopLevelNotArray
    [{**cube(4), "atoms": [atom("Cu", (0, 0, 0))]}],                    # ErrorMissingEnergy
    [cfg(4, 0.0, [{"element": "Cu", "position": [0, 0]}])],             # ErrorMalformedPosition
    "not valid json {{{",                                               # ErrorInvalidJson
])
def test_config_errors(doc):
    with pytest.raises(io.FormatError) as e:
        read(doc)
    assert str(e.value)


# ---------------------------------------------------------------------------
# PotentialReader (test_potential_reader.cpp)

def oracle_vd(t, r):
    """Value and d/dr of one parsed table at r, by the oracle."""
    if t.kind == FS_TABLE_SPLINE:
        x = np.linspace(t.rmin, t.rmax, t.values.size)
        out = O.spline_eval(x, t.values, float(r))
        return out[0], out[1]
    out, _, _ = O.form_eval(t.form, t.values, float(r), t.rmax)
    return out[0], out[1]


def oracle_sampler(model):
    def sample(k, r):
        vd = np.array([oracle_vd(model.tables[k], q) for q in np.atleast_1d(r)])
        return vd[:, 0], vd[:, 1]
    return sample


def section(fmt, pots):
    return json.dumps({"format": fmt, "potentials": pots})


def test_potential_tabulated_two_functions():  # Tabulated_TwoFunctions
    tabs = io.read_potential(section("tabulated", [{"rmin": 1.0, "rmax": 3.0, "knots": [0.5, 0.0, 0.5]},
                                                   {"rmin": 2.0, "rmax": 4.0, "knots": [1.0, 0.0, 1.0]}]))
    assert len(tabs) == 2
    assert (tabs[0].rmin, tabs[0].rmax) == (1.0, 3.0)
    assert (tabs[1].rmin, tabs[1].rmax) == (2.0, 4.0)


def test_potential_tabulated_knot_values_round_trip():  # Tabulated_KnotValuesRoundTrip
    (t,) = io.read_potential(section("tabulated", [{"rmin": 0.0, "rmax": 4.0, "knots": [2.0, 1.0, 0.0, 1.0, 2.0]}]))
    for r, want in zip((0.0, 1.0, 2.0, 3.0, 4.0), (2.0, 1.0, 0.0, 1.0, 2.0)):
        assert abs(oracle_vd(t, r)[0] - want) <= 1e-10


def test_potential_analytic_pair_lj():  # Analytic_PairLJ
    (t,) = io.read_potential(section("analytic", [{"type": "pair_lj", "rmin": 2.0, "rmax": 6.0,
                                                   "epsilon": 1.0, "sigma": 2.5}]))
    assert (t.rmin, t.rmax) == (2.0, 6.0)
    r_eq = 2.5 * 2.0 ** (1.0 / 6.0)
    v, d = oracle_vd(t, r_eq)
    assert abs(v + 1.0) <= 1e-12 and abs(d) <= 1e-10


def test_potential_analytic_morse():  # Analytic_Morse
    (t,) = io.read_potential(section("analytic", [{"type": "morse", "rmin": 1.5, "rmax": 5.0,
                                                   "De": 2.0, "a": 1.5, "re": 2.5}]))
    v, d = oracle_vd(t, 2.5)
    assert abs(v + 2.0) <= 1e-12 and abs(d) <= 1e-12


def test_potential_error_missing_format_key():  # Error_MissingFormatKey
    with pytest.raises(io.FormatError) as e:
        io.read_potential('{"potentials": []}')
    assert str(e.value)


def test_potential_error_unknown_format():  # Error_UnknownFormat
    with pytest.raises(io.FormatError, match="unsupported"):
        io.read_potential('{"format": "xyz", "potentials": []}')


def test_potential_error_unknown_analytic_function():  # Error_UnknownAnalyticFunction
    with pytest.raises(io.FormatError, match="unknown analytic function"):
        io.read_potential(section("analytic", [{"type": "born_mayer", "rmin": 1.0, "rmax": 6.0}]))


def test_potential_error_knot_not_a_number():  # Error_KnotNotANumber
    with pytest.raises(io.FormatError) as e:
        io.read_potential(section("tabulated", [{"rmin": 0.0, "rmax": 4.0, "knots": [1.0, "bad", 3.0]}]))
    assert str(e.value)


# ---------------------------------------------------------------------------
# ForceModelReader (test_force_model_reader.cpp)

def tab(rmin, rmax, knots):
    return {"rmin": rmin, "rmax": rmax, "knots": knots}


def model(doc):
    return io.read_model(json.dumps(doc))


def test_model_pair_analytic_lj():  # Pair_Analytic_LJ
    m = model({"model": "pair", "format": "analytic",
               "potentials": [{"type": "pair_lj", "rmin": 2.0, "rmax": 6.0, "epsilon": 1.0, "sigma": 2.5}]})
    assert m.family == FS_FAMILY_PAIR and len(m.tables) == 1
    v, d = oracle_vd(m.tables[0], 2.5 * 2.0 ** (1.0 / 6.0))
    assert abs(v + 1.0) <= 1e-12 and abs(d) <= 1e-10


def test_model_pair_tabulated():  # Pair_Tabulated
    m = model({"model": "pair", "format": "tabulated", "potentials": [tab(1.0, 3.0, [1.0, 0.0, 1.0])]})
    assert m.family == FS_FAMILY_PAIR and len(m.tables) == 1
    assert abs(oracle_vd(m.tables[0], 2.0)[0]) <= 1e-10


EAM_1 = {"model": "eam", "ntypes": 1,
         "pair": {"format": "tabulated", "potentials": [tab(1.5, 6.0, [2.0, 1.0, 0.0, 1.0, 2.0])]},
         "density": {"format": "tabulated", "potentials": [tab(1.5, 6.0, [1.0, 0.5, 0.0, 0.0, 0.0])]},
         "embedding": {"format": "analytic",
                       "potentials": [{"type": "sqrt", "rmin": 0.0, "rmax": 5.0, "A": -1.0, "B": 0.0}]}}


def test_model_eam_single_type_tabulated():  # EAM_SingleType_Tabulated
    m = model(EAM_1)
    assert m.family == FS_FAMILY_EAM and m.ntypes == 1
    assert abs(oracle_vd(m.tables[0], 3.75)[0]) <= 1e-2  # the middle knot
    assert oracle_vd(m.tables[1], 1.5)[0] > 0.0


def eam_2(npair=3):
    pairs = [tab(1.5, 5.0, [1.0, 0.0, 1.0]), tab(1.5, 5.0, [0.5, 0.0, 0.5]), tab(1.5, 5.0, [0.8, 0.0, 0.8])]
    return {"model": "eam", "ntypes": 2,
            "pair": {"format": "tabulated", "potentials": pairs[:npair]},
            "density": {"format": "tabulated",
                        "potentials": [tab(1.5, 5.0, [1.0, 0.5, 0.0]), tab(1.5, 5.0, [0.8, 0.4, 0.0])]},
            "embedding": {"format": "tabulated",
                          "potentials": [tab(0.0, 3.0, [0.0, -1.0, -1.5]), tab(0.0, 3.0, [0.0, -0.8, -1.2])]}}


def test_model_eam_two_types_pair_count():  # EAM_TwoTypes_PairColCount
    m = model(eam_2())
    assert m.ntypes == 2 and len(m.tables) == 3 + 2 + 2


SI_TERSOFF = {"A": 1830.8, "B": 471.18, "lambda": 2.4799, "mu": 1.7322, "beta": 1.1e-6, "n": 0.78734,
              "c": 100390.0, "d": 16.218, "h": -0.59825, "R": 2.7, "S": 3.0}


def test_model_tersoff_si_single_type():  # Tersoff_Si_SingleType
    m = model({"model": "tersoff", "ntypes": 1, "potentials": [SI_TERSOFF]})
    assert m.family == FS_FAMILY_TERSOFF and m.ntypes == 1
    v = dict(zip(TERSOFF_FIELDS, m.tables[0].values))
    assert (v["A"], v["B"], v["lambda"], v["R"], v["S"]) == (1830.8, 471.18, 2.4799, 2.7, 3.0)


def test_model_stiweb_si_single_type():  # StiWeb_Si_SingleType
    sw = {"A": 7.0496, "B": 0.6022, "p": 4.0, "q": 0.0, "delta": 2.0951, "a1": 3.7712, "gamma": 2.5141,
          "a2": 3.7712}
    m = model({"model": "stiweb", "ntypes": 1, "potentials": [sw], "lambda": [45.534]})
    assert m.family == FS_FAMILY_SW and m.ntypes == 1
    v = dict(zip(io.SW_FIELDS, m.tables[0].values))
    assert all(v[k] == sw[k] for k in ("A", "B", "delta", "a1", "gamma", "a2"))
    assert m.tables[1].values.size == 1 and m.tables[1].values[0] == 45.534


def test_model_angular_single_type():  # Angular_SingleType
    m = model({"model": "angular", "ntypes": 1,
               "pair": {"format": "analytic", "potentials": [
                   {"type": "morse", "rmin": 1.5, "rmax": 5.0, "De": 1.0, "a": 1.5, "re": 2.5}]},
               "radial": {"format": "analytic", "potentials": [
                   {"type": "exp_decay", "rmin": 1.5, "rmax": 5.0, "A": 1.0, "B": 1.0}]},
               "angular": {"format": "tabulated", "potentials": [tab(-1.0, 1.0, [0.0, -0.5, 0.0, -0.5, 0.0])]}})
    assert m.family == FS_FAMILY_ANGULAR and m.ntypes == 1


def test_model_bare_pair_section():  # BarePairSection_TreatedAsPairModel
    m = model({"format": "tabulated", "potentials": [tab(1.5, 6.0, [2.0, 1.0, 0.0, 1.0, 2.0])]})
    assert m.family == FS_FAMILY_PAIR and m.ntypes == 1


def test_model_bare_pair_section_invalid_count():  # BarePairSection_InvalidCount
    with pytest.raises(io.FormatError) as e:
        model({"format": "tabulated", "potentials": [tab(1.5, 6.0, [2.0, 1.0, 0.0]), tab(1.5, 6.0, [1.0, 0.5, 0.0])]})
    assert str(e.value)


def test_model_error_unknown_model():  # Error_UnknownModel
    with pytest.raises(io.FormatError) as e:
        model({"model": "meam", "ntypes": 1})
    assert str(e.value)


def test_model_error_eam_missing_section():  # Error_EAM_MissingSection
    doc = {k: v for k, v in EAM_1.items() if k != "embedding"}
    with pytest.raises(io.FormatError, match="embedding"):
        model(doc)


def test_model_error_eam_wrong_pair_count():  # Error_EAM_WrongPairCount
    with pytest.raises(io.FormatError) as e:
        model(eam_2(npair=1))
    assert str(e.value)


def test_model_error_tersoff_missing_param():  # Error_Tersoff_MissingParam
    with pytest.raises(io.FormatError):
        model({"model": "tersoff", "ntypes": 1, "potentials": [{"A": 1830.8, "B": 471.18}]})


def test_model_error_invalid_json():  # Error_InvalidJson
    with pytest.raises(io.FormatError) as e:
        io.read_model("not valid json {{{")
    assert str(e.value)


# global parameters: one smooth-cutoff h shared by a morse_sc pair and an
# exp_decay_sc density (kEamGlobalH)
EAM_GLOBAL_H = {
    "model": "eam", "ntypes": 1,
    "globals": {"h": {"value": 1.0, "min": 0.5, "max": 2.0}},
    "pair": {"format": "analytic", "potentials": [
        {"type": "morse_sc", "rmin": 0.0, "rmax": 6.0, "De": 0.4, "a": 1.2, "re": 2.86, "h": {"global": "h"}}]},
    "density": {"format": "analytic", "potentials": [
        {"type": "exp_decay_sc", "rmin": 0.0, "rmax": 6.0, "A": 1.0, "B": 1.0, "h": {"global": "h"}}]},
    "embedding": {"format": "analytic", "potentials": [
        {"type": "sqrt", "rmin": 0.0, "rmax": 5.0, "A": -1.0, "B": 1.0}]}}


def test_model_eam_global_h_parsed_and_counted():  # EAM_GlobalH_ParsedAndCounted
    m = model(EAM_GLOBAL_H)
    assert len(m.globals) == 1 and len(m.globals[0].links) == 2
    # morse_sc 3 (h fixed) + exp_decay_sc 2 (h fixed) + sqrt 2 + 1 global
    assert m.free_values().size == 8
    # the oracle's parameter layout agrees: tables, then the global
    o = O.Oracle()
    o.set_model(m)
    assert o.D == 8
    np.testing.assert_array_equal(o.gather_params(), m.free_values())
    lo, hi = o.gather_bounds()
    assert lo[-1] == -math.inf and hi[-1] == math.inf  # a global keeps no min/max


def test_model_eam_global_h_gather_scatter_round_trip():  # EAM_GlobalH_GatherScatterRoundTrip
    m = model(EAM_GLOBAL_H)
    x0 = m.free_values()
    np.testing.assert_array_equal(m.with_values(x0).free_values(), x0)


def test_model_eam_global_h_broadcast_reaches_all_links():  # EAM_GlobalH_BroadcastReachesAllLinks
    m = model(EAM_GLOBAL_H)
    rt = 5.5  # near the 6.0 cut-off: the switching factor of h is active
    phi0, rho0 = oracle_vd(m.tables[0], rt)[0], oracle_vd(m.tables[1], rt)[0]
    x = m.free_values()
    x[-1] = 1.7  # the global h is the last slot
    m2 = m.with_values(x)
    assert oracle_vd(m2.tables[0], rt)[0] != phi0
    assert oracle_vd(m2.tables[1], rt)[0] != rho0
    # and through the oracle's own scatter
    o = O.Oracle()
    o.set_model(m)
    o.set_params(x)
    np.testing.assert_array_equal(o.gather_params(), x)


def test_model_global_errors():
    doc = json.loads(json.dumps(EAM_GLOBAL_H))
    doc["pair"]["potentials"][0]["h"] = {"global": "nope"}
    with pytest.raises(io.FormatError, match="undefined global"):
        model(doc)
    doc = json.loads(json.dumps(EAM_GLOBAL_H))
    doc["embedding"]["potentials"][0]["A"] = {"global": "h"}
    doc["embedding"]["potentials"][0]["type"] = "sqrt"
    doc["pair"]["potentials"][0]["zz"] = {"global": "h"}
    with pytest.raises(io.FormatError, match="not valid for analytic type"):
        model(doc)


def test_model_globals_write_read_round_trip():
    m = model(EAM_GLOBAL_H)
    m2 = io.read_model(io.write_model(m))
    assert len(m2.globals) == 1 and m2.globals[0].links == m.globals[0].links
    np.testing.assert_array_equal(m2.free_values(), m.free_values())


# ---------------------------------------------------------------------------
# WriteModel (test_force_model_reader.cpp) and the pair writers

def eam_with_embedding(rmin, B):
    doc = json.loads(json.dumps(EAM_1))
    doc["embedding"]["potentials"][0].update(rmin=rmin, B=B)
    return model(doc)


def test_write_native_eam_analytic_embedding_round_trips():  # WriteModel.EAM_AnalyticEmbedding_RoundTrips
    m = eam_with_embedding(0.0, 1.0)
    text = io.write_native(m, oracle_sampler(m))
    assert "null" not in text
    back = io.read_model(text)
    assert back.family == FS_FAMILY_EAM
    # every section tabulated on 500 knots of the table's span
    assert all(t.kind == FS_TABLE_SPLINE and t.values.size == io.DEFAULT_KNOTS for t in back.tables)
    emb = back.tables[2]
    r = np.linspace(emb.rmin, emb.rmax, io.DEFAULT_KNOTS)
    np.testing.assert_allclose(emb.values, [oracle_vd(m.tables[2], q)[0] for q in r], rtol=0, atol=0)


def test_write_native_non_finite_knots_fail_loudly():  # WriteModel.NonFiniteKnots_FailsLoudly
    m = eam_with_embedding(0.5, 0.0)  # A·sqrt(ρ/B) with B = 0
    with pytest.raises(io.FormatError, match="non-finite"):
        io.write_native(m, oracle_sampler(m))


def test_write_native_ml_standardization_round_trips():  # WriteModel.ML_Standardization_RoundTrips
    from forcesmith_b200.abi import Model, Table
    spec = Table.acsf(6.0, 0, [(0.5, 0.0), (1.2, 1.5), (0.3, 2.5)], [], [], [])
    head = Table.linear_head([0.7, -0.4, 0.25], 0.1, fixed=np.array([0, 0, 0, 0], np.uint8))
    m = Model(FS_FAMILY_ACSF, 1, [spec, head]).with_standardization([[0.1, 0.2, 0.3]], [[2.0, 4.0, 0.5]])
    text = io.write_native(m, oracle_sampler(m))
    assert "standardization" in text
    back = io.read_model(text)
    np.testing.assert_allclose(back.tables[2].values, m.tables[2].values)


def pair_model():
    return model({"model": "pair", "ntypes": 2, "format": "analytic", "potentials": [
        {"type": "morse", "rmin": 1.5, "rmax": 5.0, "De": 0.5, "a": 1.3, "re": 2.6},
        {"type": "pair_lj", "rmin": 2.0, "rmax": 6.0, "epsilon": 0.2, "sigma": 2.4},
        {"type": "exp_decay", "rmin": 1.0, "rmax": 4.5, "A": 3.0, "B": 1.1}]})


def test_write_native_pair_model_is_a_bare_section():
    m = pair_model()
    back = io.read_model(io.write_native(m, oracle_sampler(m)))
    assert back.family == FS_FAMILY_PAIR and back.ntypes == 2
    assert [(t.rmin, t.rmax) for t in back.tables] == [(1.5, 5.0), (2.0, 6.0), (1.0, 4.5)]


def test_write_lammps_layout():  # output_writer.cpp:266-289
    m = pair_model()
    text = io.write_lammps(m, oracle_sampler(m))
    blocks = text.split("# pair potential ")[1:]
    assert len(blocks) == 3
    for k, b in enumerate(blocks):
        lines = b.split("\n")
        assert lines[0] == str(k) and lines[1] == f"POT_{k}"
        lo, hi = m.tables[k].rmin, m.tables[k].rmax
        assert lines[2] == f"N 500 R {lo:g} {hi:g}" and lines[3] == ""
        rows = [ln.split() for ln in lines[4:504]]
        assert [int(r[0]) for r in rows] == list(range(1, 501))
        r = np.array([float(r[1]) for r in rows])
        np.testing.assert_allclose(r, lo + np.arange(500) * (hi - lo) / 499, rtol=1e-5)
        q = 123
        v, d = oracle_vd(m.tables[k], lo + q * (hi - lo) / 499)
        assert rows[q][2] == f"{v:g}" and rows[q][3] == f"{d:g}"


def test_write_imd_layout():  # output_writer.cpp:291-310
    m = pair_model()
    lines = io.write_imd(m, oracle_sampler(m)).rstrip("\n").split("\n")
    assert lines[:3] == ["#F 3 3", "#T IMD", "#E"]
    assert lines[3:6] == [f"{t.rmin:g} {t.rmax:g} 500" for t in m.tables]
    assert len(lines) == 6 + 3 * 500
    t = m.tables[1]
    assert lines[6 + 500 + 7] == f"{oracle_vd(t, t.rmin + 7 * (t.rmax - t.rmin) / 499)[0]:g}"


def test_write_model_file_dispatch(tmp_path, capsys):  # write_model.cpp:22-55
    m = pair_model()
    s = oracle_sampler(m)
    io.write_model_file(m, tmp_path / "a.lmp", "lammps", s)
    io.write_model_file(m, tmp_path / "a.imd", "imd", s)
    assert (tmp_path / "a.lmp").read_text().startswith("# pair potential 0")
    assert (tmp_path / "a.imd").read_text().startswith("#F 3 3")
    e = eam_with_embedding(0.0, 1.0)
    io.write_model_file(e, tmp_path / "e.json", "lammps", oracle_sampler(e))
    assert "writing native JSON" in capsys.readouterr().err
    assert io.read_model(str(tmp_path / "e.json")).family == FS_FAMILY_EAM
