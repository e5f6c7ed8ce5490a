"""Ragged batches for the per-bond and per-triplet kernels (Stillinger–Weber,
Tersoff, Angular, ACSF, LMBTR): an isolated atom (no pairs, no triplets), a dimer
(pairs, no triplets), a bent trimer, and a periodic diamond cell, in one
batch, against the oracle in FP64.

Tolerances: forces, energy, stress, F rows |Δ| ≤ 1e-9·(1 + |x|); objective
1e-9 relative.  LMBTR, whose oracle forces are the reference's central
differences of the descriptor: energies 1e-10·(1 + |E|), forces and stress
1e-7 of their largest magnitude (grids and cutoff as in test_gpu_lmbtr.py).
"""
import numpy as np
import pytest

from forcesmith_b200 import synth
from forcesmith_b200.abi import FS_FAMILY_ACSF, FS_FAMILY_ANGULAR, FS_FAMILY_TERSOFF, Model, Table, acsf_size
from oracle import api as O
from tests.helpers import cluster, concat, label

pytestmark = pytest.mark.gpu


def ragged():
    iso = cluster([[0.0, 0.0, 0.0]], 20.0)
    dimer = cluster([[0.0, 0.0, 0.0], [2.3, 0.1, 0.0]], 20.0)
    trimer = cluster([[0.0, 0.0, 0.0], [2.3, 0.0, 0.0], [-0.8, 2.2, 0.3]], 20.0)
    dia = synth.diamond(1, cells=(2,), seed=83)
    return concat(iso, dimer, trimer, dia)


def models():
    r = np.linspace(1.8, 3.8, 10)
    c = np.linspace(-1.0, 1.0, 9)
    spec = Table.acsf(3.9, g1=1, g2=[(0.5, 2.3), (1.0, 3.0)], g4=[(0.05, 1.0, 1.0)], g5=[(0.08, 2.0, -1.0)])
    return {
        "sw": synth.sw_start_model(),
        "tersoff": Model(FS_FAMILY_TERSOFF, 1, [Table.tersoff(3264.7, 95.373, 3.2394, 1.3258, 0.33675, 22.956,
                                                              4.8381, 2.0417, 0.0, 3.0, 3.2)]),
        "angular": Model(FS_FAMILY_ANGULAR, 1, [
            Table.spline(1.8, 3.8, 2.0 * (np.exp(-3 * (r - 2.35)) - 2 * np.exp(-1.5 * (r - 2.35))) * (1 - (r / 3.8) ** 4)),
            Table.spline(1.8, 3.8, np.exp(-1.2 * (r - 2.35)) * (1 - (r / 3.8) ** 3)),
            Table.spline(-1.0, 1.0, 1.5 * (c + 1.0 / 3.0) ** 2)]),
        "acsf": Model(FS_FAMILY_ACSF, 1, [spec, Table.linear_head(np.linspace(0.4, -0.3, acsf_size(spec, 1)), -4.0)]),
    }


@pytest.mark.parametrize("which", ["sw", "tersoff", "angular", "acsf"])
def test_ragged_batch_fp64(which):
    from forcesmith_b200.gpu import GpuSession
    m = models()[which]
    ds = ragged()
    ds = label(ds, m.with_values(m.free_values() * 1.02), O.Oracle, 1.0, 0.2)
    g = GpuSession(0, "fp64")
    g.upload(ds)
    g.set_model(m)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(m)
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    for key in ("forces", "energy", "stress", "F"):
        a, b = np.asarray(rg[key]), np.asarray(ro[key])
        err = np.max(np.abs(a - b) / (1.0 + np.abs(b)))
        assert err <= 1e-9, (which, key, err)
    assert abs(rg["obj"] - ro["obj"]) <= 1e-9 * ro["obj"]
    assert np.all(np.abs(rg["forces"][0]) == 0.0)  # the isolated atom


def test_ragged_batch_lmbtr_fp64():
    from forcesmith_b200.gpu import GpuSession
    from tests.test_gpu_lmbtr import SMOOTH, clear_cutoff, model as lmbtr_model
    ds = ragged()
    m = lmbtr_model(1, clear_cutoff(ds, 3.6, 3.95), SMOOTH, 8)
    ds = label(ds, m.with_values(m.free_values() * 1.02), O.Oracle, 1.0, 0.2)
    g = GpuSession(0, "fp64")
    g.upload(ds)
    g.set_model(m)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(m)
    rg, ro = g.eval(1.0, 0.2), o.eval(1.0, 0.2)
    assert np.max(np.abs(rg["energy"] - ro["energy"]) / (1.0 + np.abs(ro["energy"]))) <= 1e-10
    assert np.abs(rg["forces"] - ro["forces"]).max() <= 1e-7 * np.abs(ro["forces"]).max()
    assert np.abs(rg["stress"] - ro["stress"]).max() <= 1e-7 * np.abs(ro["stress"]).max()
    assert np.all(np.abs(rg["forces"][0]) == 0.0)  # the isolated atom: no neighbours, u = 0
    assert rg["energy"][0] == m.tables[1].values[-1]  # … and its energy is the bias
