"""LMBTR descriptors with linear heads on the device against the oracle
(through the C ABI).

The oracle restates the reference, whose LMBTR forces come from central
differences (h = 1e-4) of the whole descriptor; the device differentiates
the same descriptor exactly.  Where the descriptor is smooth the two differ by
the central difference's truncation error, O(h²), far below the bars here.
The descriptor jumps where a neighbour crosses rcut or a bin crosses the edge
of a Gaussian's 5σ window; a central difference across such a jump picks up
(jump)/(2h).  So the force, stress and Jacobian cases use grids whose
Gaussians are wider than the grid (σ2 = 1.3 on [0, 6], σ3 = 0.45 on [−1, 1],
no bin ever outside 5σ) and a cutoff at least 1.5e-4 from every pair distance (a ±h move of one
component changes a distance by at most h);
the reference's default widths (σ2 = 0.3, σ3 = 0.1, windows active) are
checked on energies, which involve no difference, and on the bulk of the
force components.

Tolerances:
  energy, F energy rows      FP64 1e-10·(1 + |E|);  FP32 1e-5 relative
  forces, stress             FP64 1e-7·max|F|;      FP32 5e-5·max|F|
  Jacobian                   FP64 1e-7·max|J column| + 1e-10; FP32 1e-4·max|J column|
  lsq                        one step from a perturbed head recovers the
                             labels: objective after ≤ 1e-8 × before (FP64)
  standardization statistics FP64 1e-10, FP32 1e-5 (means) relative
"""
import numpy as np
import pytest

from forcesmith_b200 import synth
from forcesmith_b200.abi import FS_FAMILY_LMBTR, Model, Table, lmbtr_size
from oracle import api as O
from tests.helpers import label

pytestmark = pytest.mark.gpu

SMOOTH = dict(k2=(0.0, 6.0, 12, 1.3), k3=(-1.0, 1.0, 10, 0.45))
DEFAULT = dict(k2=(0.0, 6.0, 50, 0.3), k3=(-1.0, 1.0, 50, 0.1))


def clear_cutoff(ds, lo=4.1, hi=4.4):
    """A cutoff in [lo, hi] at least 1.5e-4 from every pair distance of ds."""
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model(int(ds.type.max()) + 1, hi + 0.1, SMOOTH, 0))
    r = np.sort(np.linalg.norm(o.neighbors()[2], axis=1))
    for rc in np.arange(lo, hi, 5e-5):
        k = np.searchsorted(r, rc)
        gaps = [abs(rc - r[x]) for x in (k - 1, k) if 0 <= x < r.size]
        if min(gaps) >= 1.5e-4:
            return float(rc)
    raise AssertionError("no clear cutoff")


def model(nt, rcut, grids, seed, normalize=True):
    sp = Table.lmbtr(rcut, 3.0, normalize, **grids)
    S = lmbtr_size(sp, nt)
    rng = np.random.default_rng(seed)
    return Model(FS_FAMILY_LMBTR, nt, [sp] + [Table.linear_head(rng.normal(0, 0.5, S), bias=-3.0 + t)
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


@pytest.fixture(scope="module", params=[(1, (2,), True), (2, (2, 3), True), (2, (2,), False), (2, (4,), True)],
                ids=["one", "two", "two-unnormalized", "two-512"])
def case(request):
    """two-512: a 512-atom configuration whose force-row block of J does not
    fit in shared memory, so its entries go straight to J in global memory."""
    nt, cells, norm = request.param
    ds = synth.diamond(3 if cells != (4,) else 1, cells=cells, seed=23)
    if nt == 2:
        ds.type[:] = np.random.default_rng(5).integers(0, 2, ds.type.size)
    rc = clear_cutoff(ds)
    ds = label(ds, model(nt, rc, SMOOTH, 1, norm), O.Oracle, 1.0, 0.2)
    return ds, model(nt, rc, SMOOTH, 2, norm), {}


def _oracle_jacobian(case, key, o):
    """The oracle's central-difference Jacobian, formed once per case."""
    cache = case[2]
    if key not in cache:
        cache[key] = o.jacobian_fd(1.0, 0.2)
    return cache[key]


def _energy_close(eg, eo, tol):
    eg, eo = np.asarray(eg), np.asarray(eo)
    assert np.max(np.abs(eg - eo) / (1.0 + np.abs(eo))) <= tol


def test_lmbtr_residual_fp64(case):
    ds, start, _ = case
    g, o = _pair(ds, start, "fp64")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    _energy_close(rg["energy"], ro["energy"], 1e-10)
    fmax = np.abs(ro["forces"]).max()
    assert np.abs(rg["forces"] - ro["forces"]).max() <= 1e-7 * fmax
    assert np.abs(rg["stress"] - ro["stress"]).max() <= 1e-7 * np.abs(ro["stress"]).max()
    assert abs(rg["obj"] - ro["obj"]) <= 1e-7 * ro["obj"]


def test_lmbtr_residual_fp32(case):
    ds, start, _ = case
    g, o = _pair(ds, start, "fp32")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    assert np.max(np.abs(rg["energy"] - ro["energy"]) / np.abs(ro["energy"])) <= 1e-5
    assert np.abs(rg["forces"] - ro["forces"]).max() <= 5e-5 * np.abs(ro["forces"]).max()
    assert abs(rg["obj"] - ro["obj"]) <= 1e-4 * ro["obj"]


@pytest.mark.parametrize("precision,rel,floor", [("fp64", 1e-7, 1e-10), ("fp32", 1e-4, 1e-6)])
def test_lmbtr_jacobian(case, precision, rel, floor):
    ds, start, _ = case
    g, o = _pair(ds, start, precision)
    res = g.jacobian(1.0, 0.2)
    Jf = _oracle_jacobian(case, "raw", o)
    assert res["J"].shape == Jf.shape
    bar = rel * np.abs(Jf).max(axis=0) + floor
    ratio = np.abs(res["J"] - Jf) / bar
    r, c = np.unravel_index(np.argmax(ratio), ratio.shape)
    assert ratio.max() <= 1.0, (ratio.max(), r, c, res["J"][r, c], Jf[r, c])
    F = o.eval(1.0, 0.2)["F"]
    _, Jtr = O.normal_equations(Jf, F)
    assert np.max(np.abs(res["Jtr"] - Jtr)) <= 10 * rel * np.max(np.abs(Jtr))


def test_lmbtr_lsq_step_recovers_labels(case):
    ds, start, _ = case
    g, _ = _pair(ds, start, "fp64")
    before = g.jacobian(1.0, 0.2)["obj"]
    dx = g.lsq_step(0.0)
    g.set_params(g.gather_params() + dx)
    after = g.eval(1.0, 0.2, want=("obj",))["obj"]
    assert after <= 1e-8 * before, (before, after)


def test_lmbtr_standardization(case):
    """Per-species descriptor mean and 1/σ against the oracle, then the
    residual and Jacobian of the standardized model."""
    ds, start, _ = case
    for precision, tol in (("fp64", 1e-10), ("fp32", 1e-5)):
        g, o = _pair(ds, start, precision)
        mg, ig, cg = g.acsf_standardization()
        mo, io_, co = o.acsf_standardization()
        assert cg.tolist() == co.tolist()
        np.testing.assert_allclose(mg, mo, rtol=tol, atol=tol * np.abs(mo).max())
        live = io_ > 0
        np.testing.assert_allclose(ig[live], io_[live], rtol=tol * 100, atol=0)
    m = start.with_standardization(mo, io_)
    g, o = _pair(ds, m, "fp64")
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    _energy_close(rg["energy"], ro["energy"], 1e-9)
    assert np.abs(rg["forces"] - ro["forces"]).max() <= 1e-7 * np.abs(ro["forces"]).max()
    res, Jf = g.jacobian(1.0, 0.2), _oracle_jacobian(case, "standardized", o)
    assert np.all(np.abs(res["J"] - Jf) <= 1e-7 * np.abs(Jf).max(axis=0) + 1e-9)


def test_lmbtr_default_grids():
    """The reference's default widths, windows active: energies exact; the
    central-difference window-edge jumps touch only a few force components,
    so the median and 99th percentile of |ΔF| stay at the truncation level."""
    ds = synth.diamond(2, cells=(2,), seed=31)
    ds.type[:] = np.random.default_rng(2).integers(0, 2, ds.type.size)
    rc = clear_cutoff(ds)
    m = model(2, rc, DEFAULT, 3)
    for precision, tol in (("fp64", 1e-10), ("fp32", 1e-5)):
        g, o = _pair(ds, m, precision)
        rg, ro = g.eval(1.0, 0.0), o.eval(1.0, 0.0)
        assert np.max(np.abs(rg["energy"] - ro["energy"]) / np.abs(ro["energy"])) <= tol
        d = np.abs(rg["forces"] - ro["forces"]) / np.abs(ro["forces"]).max()
        assert np.median(d) <= (1e-7 if precision == "fp64" else 5e-5)
        assert np.percentile(d, 99) <= 1e-3
