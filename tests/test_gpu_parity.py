"""Parity of the sm_100a path (called through the C ABI) with the oracle.

Tolerances (stated here, as the comparison bar):
  neighbour sets              bit-exact (counts, j, image) in the reference order
  FP64 mode  forces / stress  |Δ| ≤ 1e-9·(1 + |x|)       (bar: 1e-5 relative)
             energy, F rows   |Δ| ≤ 1e-9·(1 + |x|)
             objective        relative 1e-9
             Jacobian         vs analytic oracle 1e-9·(1 + |J|); vs the
                              reference's central differences 1e-5·|J| + 1e-8
  FP32 mode  forces           |Δ| ≤ 2e-5·max|F_ref|  (FP32 spline arithmetic;
                              pair vectors rebuilt in FP64)
             objective        relative 1e-4
             Jacobian         |Δ| ≤ 1e-4·max|J column| per column
"""
import math

import numpy as np
import pytest

from forcesmith_b200 import synth
from forcesmith_b200.abi import Model, Table, FS_FAMILY_EAM, FS_FAMILY_PAIR
from oracle import api as O
from tests.helpers import cluster, concat, label, small_ternary, ternary_models, spline_pair_model

pytestmark = pytest.mark.gpu


def _gpu(precision="fp64", lpa=0):
    from forcesmith_b200.gpu import GpuSession
    return GpuSession(0, precision, lpa)


def _pair(ds, model, precision="fp64", lpa=0):
    g = _gpu(precision, lpa)
    g.upload(ds)
    g.set_model(model)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model)
    return g, o


def _close(a, b, rel, what):
    a, b = np.asarray(a), np.asarray(b)
    err = np.max(np.abs(a - b) / (1.0 + np.abs(b))) if a.size else 0.0
    assert err <= rel, f"{what}: max rel err {err:.3e} > {rel:.1e}"


@pytest.fixture(scope="module")
def ternary_small():
    true, start = ternary_models(20)
    ds = small_ternary(6, 48, seed=99)
    ds = label(ds, true, O.Oracle, 1.0, 0.1)
    return ds, true, start


def _geometries():
    a = 3.615
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]) * a
    fcc = cluster(np.array([np.array([x, y, z]) * a + b for x in range(2) for y in range(2)
                            for z in range(2) for b in basis]), 2 * a)
    tri = cluster(np.random.default_rng(1).uniform(-3, 14, (40, 3)), 10.0)
    tri.box9[0] = [10.0, 5.0, 0.0, 0.0, 8.66, 0.0, 0.0, 0.0, 10.0]
    small = synth.packing(np.array([32, 40], np.int32), seed=5)
    mi = cluster([[0, 0, 0], [9.5, 0, 0]], 10.0)
    ds = concat(fcc, tri, small.subset([0]), small.subset([1]), mi)
    ds.type[:] = 0  # one species: the neighbour set does not depend on it
    return ds


@pytest.mark.parametrize("rcut", [1.0, 0.75 * 3.615, 6.0])
def test_neighbor_sets_bit_exact(rcut):
    ds = _geometries()
    model = Model(FS_FAMILY_PAIR, 1, [Table.spline(0.0, rcut, np.zeros(4))])
    g, o = _pair(ds, model)
    assert g.num_pairs() == o.num_pairs()
    assert np.array_equal(g.neighbor_counts(ds.n_atoms), o.neighbor_counts(ds.n_atoms))
    gj, gimg = g.neighbors()
    oj, oimg, _ = o.neighbors()
    assert np.array_equal(gj, oj)
    assert np.array_equal(gimg, oimg)


def test_neighbor_sets_ternary_bit_exact(ternary_small):
    ds, true, _ = ternary_small
    g, o = _pair(ds, true)
    gj, gimg = g.neighbors()
    oj, oimg, _ = o.neighbors()
    assert np.array_equal(gj, oj) and np.array_equal(gimg, oimg)


@pytest.mark.parametrize("lpa", [0, 4, 8, 16, 32])
def test_eam_residual_fp64(ternary_small, lpa):
    ds, _, start = ternary_small
    g, o = _pair(ds, start, "fp64", lpa)
    rg, ro = g.eval(1.0, 0.1), o.eval(1.0, 0.1)
    _close(rg["forces"], ro["forces"], 1e-9, "forces")
    _close(rg["energy"], ro["energy"], 1e-9, "energy")
    _close(rg["stress"], ro["stress"], 1e-9, "stress")
    _close(rg["F"], ro["F"], 1e-9, "F")
    assert abs(rg["obj"] - ro["obj"]) <= 1e-9 * ro["obj"]


def test_eam_residual_fp32(ternary_small):
    ds, _, start = ternary_small
    g, o = _pair(ds, start, "fp32")
    rg, ro = g.eval(1.0, 0.1), o.eval(1.0, 0.1)
    scale = np.max(np.abs(ro["forces"]))
    assert np.max(np.abs(rg["forces"] - ro["forces"])) <= 2e-5 * scale
    assert abs(rg["obj"] - ro["obj"]) <= 1e-4 * ro["obj"]
    assert np.max(np.abs(rg["energy"] - ro["energy"]) / np.abs(ro["energy"])) <= 1e-5


def test_pair_residual_half_open_gate():
    ds = small_ternary(3, 40, seed=12)
    ds.type[:] = ds.type % 2
    model = spline_pair_model(2, rmax=5.5)
    ds = label(ds, model.with_values(model.free_values() * 1.02), O.Oracle, 1.0, 0.3)
    g, o = _pair(ds, model)
    rg, ro = g.eval(1.0, 0.3), o.eval(1.0, 0.3)
    _close(rg["F"], ro["F"], 1e-9, "F")


def test_eam_clamp_limit_rows():
    """ρ beyond the embedding span: limit rows and the clamped embedding
    (kernels.hpp:19-31; eam_force.cpp:151-190)."""
    true, start = ternary_models(12)
    ds = small_ternary(3, 40, seed=21)
    for t in start.tables[9:]:  # shrink the embedding span below the observed ρ
        t.rmax = 9.0
    g, o = _pair(ds, start)
    rg, ro = g.eval(1.0, 0.0), o.eval(1.0, 0.0)
    assert np.all(ro["limit"] > 0)
    _close(rg["limit"], ro["limit"], 1e-9, "limit")
    _close(rg["F"], ro["F"], 1e-9, "F")
    jg = g.jacobian(1.0, 0.0)["J"]
    ja = o.jacobian_analytic(1.0, 0.0)
    _close(jg, ja, 1e-8, "J with clamped atoms")


def test_eam_jacobian_fp64_vs_oracle(ternary_small):
    ds, _, start = ternary_small
    sub = ds.subset([0, 1])
    g, o = _pair(sub, start, "fp64")
    res = g.jacobian(1.0, 0.1)
    Ja = o.jacobian_analytic(1.0, 0.1)
    _close(res["J"], Ja, 1e-9, "J vs analytic oracle")
    Jf = o.jacobian_fd(1.0, 0.1)
    assert np.all(np.abs(res["J"] - Jf) <= 1e-5 * np.abs(Jf) + 1e-8 + 1e-6 * np.abs(Jf).max())
    F = o.eval(1.0, 0.1)["F"]
    JtJ, Jtr = O.normal_equations(Ja, F)
    _close(res["JtJ"], JtJ, 1e-9, "JtJ")
    _close(res["Jtr"], Jtr, 1e-9, "Jtr")
    assert abs(res["obj"] - float(F @ F)) <= 1e-9 * float(F @ F)


def test_eam_jacobian_fp32(ternary_small):
    ds, _, start = ternary_small
    sub = ds.subset([0, 1, 2])
    g, o = _pair(sub, start, "fp32")
    res = g.jacobian(1.0, 0.1)
    Ja = o.jacobian_analytic(1.0, 0.1)
    colmax = np.abs(Ja).max(axis=0) + 1e-30
    err = np.max(np.abs(res["J"] - Ja) / colmax)
    assert err <= 1e-4, err
    F = o.eval(1.0, 0.1)["F"]
    JtJ, Jtr = O.normal_equations(Ja, F)
    d = np.sqrt(np.outer(np.diag(JtJ), np.diag(JtJ)))
    d = d + 1e-12 * d.max()  # columns of pair types absent from the sample are zero
    rel = np.abs(res["JtJ"] - JtJ) / d
    a, b = np.unravel_index(np.argmax(rel), rel.shape)
    assert rel[a, b] <= 1e-3, (rel[a, b], a, b, res["JtJ"][a, b], JtJ[a, b])
    assert np.max(np.abs(res["Jtr"] - Jtr)) <= 1e-4 * np.max(np.abs(Jtr))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_eam_jacobian_two_ctas_per_configuration(precision):
    """20 configurations of 24 atoms fill the SMs' waves better as 40 CTAs, so
    the force-row pass gives each configuration two CTAs (alternate strides of
    its atoms) and a combine kernel adds their energy, stress and Jᵀr sums: one
    launch more per step than 6 configurations take.  Against the analytic
    oracle: FP64 J, JᵀJ, Jᵀr 1e-9·(1 + |x|); FP32 J 1e-4·max|J column|, JᵀJ
    1e-3 of √(JᵀJ_aa·JᵀJ_bb), Jᵀr 1e-4 of its largest entry."""
    from forcesmith_b200.gpu import launch_count
    true, start = ternary_models(20)
    ds = label(small_ternary(20, 24, seed=12), true, O.Oracle, 1.0, 0.1)
    per_step = []
    for sub in (ds, ds.subset(list(range(6)))):
        g = _gpu(precision)
        g.upload(sub)
        g.set_model(start)
        g.jacobian_async(1.0, 0.1)
        n0 = launch_count(g)
        g.jacobian_async(1.0, 0.1)
        per_step.append(launch_count(g) - n0)
    assert per_step[0] == per_step[1] + 1, per_step
    g, o = _pair(ds, start, precision)
    res = g.jacobian(1.0, 0.1)
    Ja = o.jacobian_analytic(1.0, 0.1)
    F = o.eval(1.0, 0.1)["F"]
    JtJ, Jtr = O.normal_equations(Ja, F)
    if precision == "fp64":
        _close(res["J"], Ja, 1e-9, "J vs analytic oracle")
        _close(res["JtJ"], JtJ, 1e-9, "JtJ")
        _close(res["Jtr"], Jtr, 1e-9, "Jtr")
    else:
        colmax = np.abs(Ja).max(axis=0) + 1e-30
        assert np.max(np.abs(res["J"] - Ja) / colmax) <= 1e-4
        d = np.sqrt(np.outer(np.diag(JtJ), np.diag(JtJ)))
        d = d + 1e-12 * d.max()
        assert np.max(np.abs(res["JtJ"] - JtJ) / d) <= 1e-3
        assert np.max(np.abs(res["Jtr"] - Jtr)) <= 1e-4 * np.max(np.abs(Jtr))


def test_pair_jacobian_fp64():
    ds = small_ternary(2, 40, seed=13)
    ds.type[:] = ds.type % 2
    model = spline_pair_model(2)
    ds = label(ds, model.with_values(model.free_values() * 1.03), O.Oracle, 1.0, 0.2)
    g, o = _pair(ds, model)
    res = g.jacobian(0.7, 0.2)
    _close(res["J"], o.jacobian_analytic(0.7, 0.2), 1e-9, "pair J")


@pytest.mark.parametrize("nknots", [48, 49])
def test_pair_jacobian_fp32_gram_paths(nknots):
    """D = 48 free knots: column-major J and the small-D JᵀJ kernel; D = 49:
    row-major J and the tensor-core JᵀJ.  J against the analytic oracle
    (1e-4·max|J column|); JᵀJ against the returned J in FP64 (1e-5 of
    √(JᵀJ_aa·JᵀJ_bb)), Jᵀr against the returned J and F (1e-5 of its largest
    entry)."""
    model = spline_pair_model(1, nknots)
    assert model.free_values().size == nknots
    ds = small_ternary(4, 40, seed=17)
    ds.type[:] = 0
    ds = label(ds, model.with_values(model.free_values() * 1.03), O.Oracle, 1.0, 0.2)
    g, o = _pair(ds, model, "fp32")
    res = g.jacobian(1.0, 0.2)
    Ja = o.jacobian_analytic(1.0, 0.2)
    colmax = np.abs(Ja).max(axis=0) + 1e-30
    assert np.max(np.abs(res["J"] - Ja) / colmax) <= 1e-4
    J = np.asarray(res["J"], np.float64)
    JtJ, Jtr = J.T @ J, J.T @ np.asarray(res["F"], np.float64)
    d = np.sqrt(np.outer(np.diag(JtJ), np.diag(JtJ)))
    d = d + 1e-12 * d.max()
    assert np.max(np.abs(res["JtJ"] - JtJ) / d) <= 1e-5
    assert np.max(np.abs(res["Jtr"] - Jtr)) <= 1e-5 * np.max(np.abs(Jtr))


def test_lm_and_lsq_steps_fp64(ternary_small):
    ds, _, start = ternary_small
    g = _gpu("fp64")
    g.upload(ds)
    g.set_model(start)
    res = g.jacobian(1.0, 0.1, want_J=False)
    for lam, mode in ((1e-3, 0), (1e-2, 1), (10.0, 0)):
        dx = g.lm_step(lam, mode)
        ref = O.lm_step(res["JtJ"], res["Jtr"], lam, mode)
        _close(dx, ref, 1e-8, f"lm_step λ={lam}")
    dx = g.lsq_step(0.0)
    _close(dx, O.lsq_step(res["JtJ"], res["Jtr"], 0.0), 1e-6, "lsq_step")


def test_population_objective(ternary_small):
    ds, _, start = ternary_small
    g, o = _pair(ds.subset([0, 1, 2]), start, "fp64")
    x0 = g.gather_params()
    xs = np.stack([x0 * synth.uniform(x0.size, 0.98, 1.02, 100 + k) for k in range(5)])
    og = g.eval_population(xs, 1.0, 0.1)
    oo = o.eval_population(xs, 1.0, 0.1)
    _close(og, oo, 1e-9, "population objective")


def _two_grid_model(start):
    """The ternary start model with its density tables on [1.8, 5.5] instead
    of the pair tables' [1.8, 6.0]: no knot grid shared by all r-functions."""
    tabs = list(start.tables)
    for a in range(3):
        tabs[6 + a] = Table.spline(tabs[6 + a].rmin, 5.5, tabs[6 + a].values)
    return Model(FS_FAMILY_EAM, 3, tabs)


@pytest.mark.parametrize("family", ["eam", "pair", "eam_two_grids"])
def test_population_objective_fp32_lanes(ternary_small, family):
    """FP32 population path (one lane per trial vector): against the FP64
    oracle (relative 1e-4, the FP32 objective bar) and against the FP32
    single-vector residual path (relative 1e-5); NP = 37 leaves a partial
    tile of trials.  "eam": the pair and density tables share a knot grid, so
    the kernel walks the sorted pair runs; "eam_two_grids" and "pair": it
    walks the neighbour list."""
    ds, _, start = ternary_small
    model = {"eam": start, "pair": spline_pair_model(3, 14), "eam_two_grids": _two_grid_model(start)}[family]
    g, o = _pair(ds.subset([0, 1, 2, 3]), model, "fp32")
    x0 = g.gather_params()
    xs = np.stack([x0 * synth.uniform(x0.size, 0.97, 1.03, 200 + k) for k in range(37)])
    og = g.eval_population(xs, 1.0, 0.1)
    oo = o.eval_population(xs, 1.0, 0.1)
    _close(og, oo, 1e-4, "population objective vs oracle")
    single = []
    for x in xs[:5]:
        g.set_params(x)
        single.append(g.eval(1.0, 0.1, want=("obj",))["obj"])
    np.testing.assert_allclose(og[:5], single, rtol=1e-5)
    assert np.array_equal(og, g.eval_population(xs, 1.0, 0.1)), "deterministic"


def test_gradient_directional_full_size():
    """Size-independent property at the full ternary workload (500 × 256):
    d/dε ‖F(x + εv)‖² = 2 vᵀJᵀF, with J from the FP32 analytic path and the
    objective from the FP64 path."""
    true, start = ternary_models(20)
    ds = synth.ternary_geometry()
    g64 = _gpu("fp64")
    g64.upload(ds)
    g64.set_model(true)
    lab = g64.eval(1.0, 0.1)
    ds = ds.with_labels(lab["forces"], lab["energy"], lab["stress"])
    g64.set_references(ds)
    g64.set_model(start)
    g32 = _gpu("fp32")
    g32.upload(ds)
    g32.set_model(start)
    res = g32.jacobian(1.0, 0.1, want_J=False)
    x = g64.gather_params()
    v = synth.uniform(x.size, -1.0, 1.0, 77)
    eps = 1e-6  # makima's |·| kinks make larger steps inexact (1e-4 is off by ~1 %)
    g64.set_params(x + eps * v)
    op = g64.eval(1.0, 0.1, want=("obj",))["obj"]
    g64.set_params(x - eps * v)
    om = g64.eval(1.0, 0.1, want=("obj",))["obj"]
    fd = (op - om) / (2 * eps)
    an = 2.0 * float(v @ res["Jtr"])
    assert abs(fd - an) <= 2e-4 * abs(fd), (fd, an)
    assert np.allclose(res["JtJ"], res["JtJ"].T, rtol=0, atol=1e-12 * np.abs(res["JtJ"]).max())
    assert np.all(np.linalg.eigvalsh(res["JtJ"]) > -1e-8 * np.abs(res["JtJ"]).max())


# ---------------------------------------------------------------- SW ---

@pytest.fixture(scope="module")
def sw_case():
    from tests.helpers import small_diamond
    ds = small_diamond(4, (2, 3), seed=31)
    ds = label(ds, synth.sw_model(), O.Oracle, 1.0, 0.2)
    return ds, synth.sw_start_model()


def test_sw_residual_fp64(sw_case):
    ds, start = sw_case
    g, o = _pair(ds, start, "fp64")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    _close(rg["forces"], ro["forces"], 1e-9, "SW forces")
    _close(rg["F"], ro["F"], 1e-9, "SW F")
    assert abs(rg["obj"] - ro["obj"]) <= 1e-9 * ro["obj"]


def test_sw_residual_fp32(sw_case):
    ds, start = sw_case
    g, o = _pair(ds, start, "fp32")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    assert np.max(np.abs(rg["forces"] - ro["forces"])) <= 2e-5 * np.max(np.abs(ro["forces"]))
    assert abs(rg["obj"] - ro["obj"]) <= 1e-4 * ro["obj"]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-5), ("fp32", 2e-3)])
def test_sw_jacobian_vs_central_differences(sw_case, precision, tol):
    """The analytic SW Jacobian against the reference's own method for SW —
    central differences (stiweb has no analytic Jacobian in the reference)."""
    ds, start = sw_case
    g, o = _pair(ds, start, precision)
    res = g.jacobian(1.0, 0.2)
    Jf = o.jacobian_fd(1.0, 0.2)
    colmax = np.abs(Jf).max(axis=0)
    err = np.abs(res["J"] - Jf) / (tol * np.abs(Jf) + 1e-8 + 1e-7 * colmax)
    assert err.max() <= 1.0, err.max()
    F = o.eval(1.0, 0.2)["F"]
    JtJ, Jtr = O.normal_equations(Jf, F)
    assert np.max(np.abs(res["Jtr"] - Jtr)) <= 10 * tol * np.max(np.abs(Jtr))


def binary_sw_model():
    """Two species: three pair slots with their own (A, B, δ, a1, γ, a2)
    (p, q fixed) and six λ_{i;jk}, one of them fixed — triplets whose ends sit
    in different slots, and columns that change from one triplet to the next."""
    from forcesmith_b200.abi import Model, Table, FS_FAMILY_SW
    base = synth.sw_model().tables[0].values
    tabs = []
    for s, f in enumerate((1.0, 0.93, 1.06)):
        v = base * np.array([f, 2.0 - f, 1, 1, f, 1.0 + 0.02 * s, 1.0 - 0.03 * s, 1.0 + 0.01 * s])
        tabs.append(Table.sw(*v, fixed=np.array([0, 0, 1, 1, 0, 0, 0, 0], np.uint8)))
    lam = 45.5 * np.array([1.0, 0.8, 1.2, 0.9, 1.1, 0.7])
    tabs.append(Table.lam(lam, fixed=np.array([0, 0, 1, 0, 0, 0], np.uint8)))
    return Model(FS_FAMILY_SW, 2, tabs)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-5), ("fp32", 2e-3)])
def test_sw_binary_residual_and_jacobian(precision, tol):
    from tests.helpers import small_diamond
    ds = small_diamond(3, (2, 3), seed=37)
    ds.type[:] = np.random.default_rng(5).integers(0, 2, ds.type.size)
    model = binary_sw_model()
    ds = label(ds, model.with_values(model.free_values() * 1.03), O.Oracle, 1.0, 0.2)
    g, o = _pair(ds, model, precision)
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    ftol = 1e-9 if precision == "fp64" else 2e-5
    assert np.max(np.abs(rg["forces"] - ro["forces"])) <= ftol * np.max(np.abs(ro["forces"]))
    assert abs(rg["obj"] - ro["obj"]) <= (1e-9 if precision == "fp64" else 1e-4) * ro["obj"]
    res = g.jacobian(1.0, 0.2)
    Jf = o.jacobian_fd(1.0, 0.2)
    assert res["J"].shape == Jf.shape and Jf.shape[1] == 3 * 6 + 5
    colmax = np.abs(Jf).max(axis=0)
    err = np.abs(res["J"] - Jf) / (tol * np.abs(Jf) + 1e-8 + 1e-7 * colmax)
    assert err.max() <= 1.0, err.max()


# --------------------------------------------------------------- ADP ---

def test_adp_residual_fp64():
    """ADP residual against the oracle (its exact Jacobian: test_gpu_adp.py)."""
    from tests.helpers import adp_spline_model
    ds = small_ternary(3, 32, seed=41)
    ds.type[:] = ds.type % 2
    model = adp_spline_model(2)
    ds = label(ds, model.with_values(model.free_values() * 1.02), O.Oracle, 1.0, 0.1)
    g, o = _pair(ds, model, "fp64")
    rg, ro = g.eval(1.0, 0.1), o.eval(1.0, 0.1)
    _close(rg["forces"], ro["forces"], 1e-9, "ADP forces")
    _close(rg["energy"], ro["energy"], 1e-9, "ADP energy")
    _close(rg["F"], ro["F"], 1e-9, "ADP F")


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_autotune_keeps_results(ternary_small, precision):
    """fs_gpu_autotune picks schedules from its candidate sets; results after
    tuning equal the untuned ones up to summation order (FP64 1e-12
    relative; FP32 at its stated bars)."""
    ds, _, start = ternary_small
    g, _ = _pair(ds, start, precision)
    before = g.eval(1.0, 0.1)
    jb = g.jacobian(1.0, 0.1, want_J=False)
    x0 = g.gather_params()
    xs = np.stack([x0 * synth.uniform(x0.size, 0.98, 1.02, 300 + k) for k in range(5)])
    pb = g.eval_population(xs, 1.0, 0.1)
    rep = g.autotune(1.0, 0.1)
    assert rep["lanes_per_atom"] in (4, 8, 16, 32)
    assert rep["k2_warps"] in ((4, 6, 8) if precision == "fp64" else (4, 6, 8, 10, 11))
    assert rep["pop_waves"] in ((2, 4, 8) if precision == "fp32" else (0,))
    after = g.eval(1.0, 0.1)
    ja = g.jacobian(1.0, 0.1, want_J=False)
    pa = g.eval_population(xs, 1.0, 0.1)
    tol = 1e-12 if precision == "fp64" else 1e-4
    _close(after["F"], before["F"], tol if precision == "fp64" else 1e-5, "F")
    assert abs(after["obj"] - before["obj"]) <= tol * abs(before["obj"])
    np.testing.assert_allclose(ja["JtJ"], jb["JtJ"], rtol=tol if precision == "fp64" else 1e-3,
                               atol=(1e-12 if precision == "fp64" else 1e-3) * np.abs(jb["JtJ"]).max())
    np.testing.assert_allclose(pa, pb, rtol=tol)


@pytest.mark.parametrize("precision,family", [("fp32", "eam"), ("fp64", "eam"), ("fp32", "sw")])
def test_copy_jacobian_rows(ternary_small, precision, family):
    """fs_gpu_copy_jacobian_rows (the row block a cached-Jacobian calculator
    writes per configuration into Eigen's column-major fjac): every
    configuration's block, copied into a larger leading dimension, equals
    the matching rows of fs_gpu_eval_jacobian's J, bit for bit.  Layouts:
    FP32 EAM row-major on the device, FP64 column-major, FP32 SW
    column-major.  Rows past the residual count are refused."""
    if family == "eam":
        ds, _, model = ternary_small
        w_s = 0.1
    else:
        from tests.helpers import small_diamond
        ds = label(small_diamond(3, (2, 3), seed=31), synth.sw_model(), O.Oracle, 1.0, 0.2)
        model, w_s = synth.sw_start_model(), 0.2
    g = _gpu(precision)
    g.upload(ds)
    g.set_model(model)
    J = g.jacobian(1.0, w_s)["J"]
    m = J.shape[0]
    extra = 2 + (6 if w_s > 0 else 0)
    r0 = 0
    for n in ds.natoms:
        rows = 3 * int(n) + extra
        blk, buf = g.jacobian_rows(r0, rows, ld=rows + 5)
        assert np.array_equal(blk, J[r0:r0 + rows])
        assert np.all(np.isnan(buf[:, rows:]))  # nothing written past the block
        r0 += rows
    assert r0 == m
    from forcesmith_b200.abi import FsError
    with pytest.raises(FsError):
        g.jacobian_rows(m - 2, 3)
