"""ACSF descriptors with linear heads on the device against the oracle
(through the C ABI).

Tolerances:
  FP64  forces, energy, stress, F rows   |Δ| ≤ 1e-9·(1 + |x|); objective 1e-9 relative
  FP32  forces                           |Δ| ≤ 2e-5·max|F|;    objective 1e-4 relative
  Jacobian (exact on the device; the oracle's central differences are exact
  up to rounding, the model being linear in its coefficients: noise
  ≈ 1e-16·|F| / 2h with h = 1e-5)
        FP64 |ΔJ| ≤ 1e-6·max|J column| + 1e-9;  FP32 |ΔJ| ≤ 1e-4·max|J column|
  lsq   one normal-equations step from a perturbed head recovers the labels:
        objective after ≤ 1e-8 × objective before (FP64)
"""
import numpy as np
import pytest

from forcesmith_b200 import synth
from forcesmith_b200.abi import FS_FAMILY_ACSF, Model, Table, acsf_size
from oracle import api as O
from tests.helpers import label

pytestmark = pytest.mark.gpu

SPEC = Table.acsf(4.2, g1=1, g2=[(0.5, 2.3), (1.0, 3.0), (2.0, 3.8), (0.3, 0.0)], g3=[1.1],
                  g4=[(0.05, 1.0, 1.0), (0.05, 2.0, -1.0)], g5=[(0.08, 1.5, 1.0)])


def model(nt, seed):
    S = acsf_size(SPEC, nt)
    rng = np.random.default_rng(seed)
    return Model(FS_FAMILY_ACSF, nt, [SPEC] + [Table.linear_head(rng.normal(0, 0.3, S), bias=-3.0 + t)
                                               for t in range(nt)])


def _pair(ds, m, precision):
    from forcesmith_b200.gpu import GpuSession
    g = GpuSession(0, precision)
    g.upload(ds)
    g.set_model(m)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(m)
    return g, o


def _close(a, b, rel, what):
    err = np.max(np.abs(np.asarray(a) - np.asarray(b)) / (1.0 + np.abs(np.asarray(b))))
    assert err <= rel, f"{what}: {err:.3e}"


@pytest.fixture(scope="module", params=[(1, (2, 3)), (2, (2, 3)), (2, (4,))], ids=["one", "two", "two-512"])
def case(request):
    """two-512: a 512-atom configuration whose J block (1543 × 42) does not
    fit in shared memory, so its terms go straight to J in global memory."""
    nt, cells = request.param
    ds = synth.diamond(4 if cells != (4,) else 1, cells=cells, seed=71)
    if nt == 2:
        ds.type[:] = np.random.default_rng(9).integers(0, 2, ds.type.size)
    ds = label(ds, model(nt, 1), O.Oracle, 1.0, 0.2)
    return ds, model(nt, 2)


def test_acsf_residual_fp64(case):
    ds, start = case
    g, o = _pair(ds, start, "fp64")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    _close(rg["forces"], ro["forces"], 1e-9, "forces")
    _close(rg["energy"], ro["energy"], 1e-9, "energy")
    _close(rg["stress"], ro["stress"], 1e-9, "stress")
    _close(rg["F"], ro["F"], 1e-9, "F")
    assert abs(rg["obj"] - ro["obj"]) <= 1e-9 * ro["obj"]


def test_acsf_residual_fp32(case):
    ds, start = case
    g, o = _pair(ds, start, "fp32")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    assert np.max(np.abs(rg["forces"] - ro["forces"])) <= 2e-5 * np.max(np.abs(ro["forces"]))
    assert abs(rg["obj"] - ro["obj"]) <= 1e-4 * ro["obj"]


@pytest.mark.parametrize("precision,rel,floor", [("fp64", 1e-6, 1e-9), ("fp32", 1e-4, 0.0)])
def test_acsf_jacobian(case, precision, rel, floor):
    ds, start = case
    g, o = _pair(ds, start, precision)
    res = g.jacobian(1.0, 0.2)
    Jf = o.jacobian_fd(1.0, 0.2)
    assert res["J"].shape == Jf.shape
    colmax = np.abs(Jf).max(axis=0)
    bar = rel * colmax + floor + 1e-30
    ratio = np.abs(res["J"] - Jf) / bar
    r, c = np.unravel_index(np.argmax(ratio), ratio.shape)
    assert ratio.max() <= 1.0, (ratio.max(), r, c, res["J"][r, c], Jf[r, c])
    F = o.eval(1.0, 0.2)["F"]
    _, Jtr = O.normal_equations(Jf, F)
    assert np.max(np.abs(res["Jtr"] - Jtr)) <= 10 * rel * np.max(np.abs(Jtr))


def test_acsf_lsq_step_recovers_labels(case):
    """NormalEquationsSolver on the device (the reference's lsq for linear
    heads): one step from the perturbed head to the labelling head."""
    ds, start = case
    g, _ = _pair(ds, start, "fp64")
    before = g.jacobian(1.0, 0.2)["obj"]
    dx = g.lsq_step(0.0)
    g.set_params(g.gather_params() + dx)
    after = g.eval(1.0, 0.2, want=("obj",))["obj"]
    assert after <= 1e-8 * before, (before, after)


# ---- feature standardization (MLBase, ml_force.hpp:607-688)

def test_acsf_standardization_statistics(case):
    """Per-species descriptor mean and 1/σ over every atom against the oracle:
    FP64 1e-10 relative, FP32 descriptors 1e-5 relative (mean) and 1e-4
    (1/σ) (sums in FP64)."""
    ds, start = case
    for precision, tol in (("fp64", 1e-10), ("fp32", 1e-5)):
        g, o = _pair(ds, start, precision)
        mg, ig, cg = g.acsf_standardization()
        mo, io_, co = o.acsf_standardization()
        assert cg.tolist() == co.tolist()
        np.testing.assert_allclose(mg, mo, rtol=tol, atol=tol * np.abs(mo).max())
        np.testing.assert_allclose(ig, io_, rtol=tol * 10, atol=0)


def _standardized(ds, start):
    o = O.Oracle()
    o.upload(ds)
    o.set_model(start)
    mean, inv_std, _ = o.acsf_standardization()
    return start.with_standardization(mean, inv_std)


def test_acsf_standardized_residual(case):
    """With standardization tables: FP64 forces, energy, stress, F rows
    1e-9·(1 + |x|); FP32 forces 2e-5·max|F|, objective 1e-4."""
    ds, start = case
    m = _standardized(ds, start)
    g, o = _pair(ds, m, "fp64")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    for key in ("forces", "energy", "stress", "F"):
        _close(rg[key], ro[key], 1e-9, key)
    g, o = _pair(ds, m, "fp32")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    assert np.max(np.abs(rg["forces"] - ro["forces"])) <= 2e-5 * np.max(np.abs(ro["forces"]))
    assert abs(rg["obj"] - ro["obj"]) <= 1e-4 * ro["obj"]


@pytest.mark.parametrize("precision,rel,floor", [("fp64", 1e-6, 1e-9), ("fp32", 1e-4, 0.0)])
def test_acsf_standardized_jacobian(case, precision, rel, floor):
    """The exact Jacobian of a standardized head (columns of w scaled by
    inv_std, energy rows shifted by −inv_std·mean per atom) against the
    oracle's central differences, with the bars of test_acsf_jacobian.

    FP32, energy rows: entry (c, w_k of species t) is Σ_i inv_std_k·D_ik −
    inv_std_k·mean_k·N_t over the configuration's atoms of species t, a
    difference of two terms of size ≈ inv_std_k·|mean_k|·N_t that cancel when
    mean is the configuration's own mean.  FP32 descriptors (a few ulp each)
    leave an error proportional to that size, so these entries are held to
    1e-5 of it (the device sums them in FP64)."""
    ds, start = case
    m = _standardized(ds, start)
    g, o = _pair(ds, m, precision)
    res = g.jacobian(1.0, 0.2)
    Jf = o.jacobian_fd(1.0, 0.2)
    bar = rel * np.abs(Jf).max(axis=0) + floor + 1e-30
    bar = np.broadcast_to(bar, Jf.shape).copy()
    if precision == "fp32":
        nt = start.ntypes
        mean, inv_std, _ = o.acsf_standardization()
        S = mean.shape[1]
        row, a0 = 0, 0
        for c in range(ds.n_cfg):
            n = int(ds.natoms[c])
            types = ds.type[a0:a0 + n]
            a0 += n
            rE = row + 3 * n
            for t in range(nt):
                cancelled = inv_std[t] * np.abs(mean[t]) * np.count_nonzero(types == t)
                bar[rE, t * S:(t + 1) * S] = np.maximum(bar[rE, t * S:(t + 1) * S], 1e-5 * cancelled)
            row += 3 * n + 8
    ratio = np.abs(res["J"] - Jf) / bar
    r, c = np.unravel_index(np.argmax(ratio), ratio.shape)
    assert ratio.max() <= 1.0, (ratio.max(), r, c, res["J"][r, c], Jf[r, c])


def test_acsf_three_species_remapped():
    """A three-species model made by species re-ranking ([A, B] → [A, B, C],
    MLBase::remap) on configurations of all three species: FP64 residual rows
    against the oracle 1e-9·(1 + |x|), and the exact FP64 Jacobian against the
    oracle's central differences (1e-6·max|J column| + 1e-9)."""
    ds = synth.diamond(3, cells=(2,), seed=17)
    ds.type[:] = np.random.default_rng(5).integers(0, 3, ds.type.size)
    m2 = model(2, 3)
    m3 = m2.acsf_remapped(["A", "B"], ["A", "B", "C"])
    rng = np.random.default_rng(6)
    for t in m3.tables[1:]:
        t.values[:-1] += rng.normal(0, 0.05, t.values.size - 1)  # every channel in use
    ds = label(ds, m3, O.Oracle, 1.0, 0.2)
    start = m3.with_values(m3.free_values() * 1.05)
    g, o = _pair(ds, start, "fp64")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    for key in ("forces", "energy", "stress", "F"):
        _close(rg[key], ro[key], 1e-9, key)
    res = g.jacobian(1.0, 0.2)
    Jf = o.jacobian_fd(1.0, 0.2)
    bar = 1e-6 * np.abs(Jf).max(axis=0) + 1e-9
    assert np.max(np.abs(res["J"] - Jf) / bar) <= 1.0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_acsf_standardization_dead_features(precision):
    """Three identical dimers: every atom sees the same environment, so every
    feature has no variance, inv_std is 0 (compute_standardization) and the
    standardized head reduces to its bias.  Statistics, residual and Jacobian against the
    oracle: the J columns of w vanish except for the energy row's mean
    shift, which cancels Σ_i D_i exactly here (|J| ≤ 1e-6 in FP32, 1e-12 in
    FP64); forces 1e-9 (FP64) / 1e-6 (FP32) absolute."""
    from tests.helpers import cluster, concat
    ds = concat(*[cluster([[0.0, 0.0, 0.0], [2.4, 0.0, 0.0]], 20.0) for _ in range(3)])
    ds = label(ds, model(1, 1), O.Oracle, 1.0, 0.2)
    start = model(1, 2)
    g, o = _pair(ds, start, precision)
    mg, ig, _ = g.acsf_standardization()
    assert np.all(ig == 0.0), ig
    m = start.with_standardization(mg, ig)
    g, o = _pair(ds, m, precision)
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    tol = 1e-9 if precision == "fp64" else 1e-6
    assert np.max(np.abs(rg["forces"])) <= tol and np.max(np.abs(ro["forces"])) <= 1e-12
    _close(rg["energy"], ro["energy"], tol, "energy")
    res = g.jacobian(1.0, 0.2)
    assert np.max(np.abs(res["J"])) <= (1e-12 if precision == "fp64" else 1e-6)
