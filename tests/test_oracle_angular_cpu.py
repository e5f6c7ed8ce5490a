"""The oracle's Angular restatement, pinned against the reference's unit
tests (tests/unit/test_angular_force.cpp): LJ pair (ε = σ = 1, span
[0.1, 20]), radial f = e^{−r} (span [0, 20]), angular g = (cos θ + ½)²,
an equilateral triangle of side 2.5 Å and a dimer in a 100 Å box.

  NewtonThirdLaw_Triangle / _Dimer        1e-11 / 1e-12
  ZeroFModZerosThreeBody                  f ≡ 0 reproduces the pair-only model, 1e-12
  EnergyIsFinite, ForcesIdempotent        1e-14
  ForceConsistentWithEnergyFD             F_x(0) = −dE/dx₀, h = 1e-5 Å, 1e-5 rel
  StressSymmetric                         1e-13
"""
import numpy as np

from forcesmith_b200.abi import FS_FAMILY_ANGULAR, FS_FAMILY_PAIR, Model, Table
from oracle import api as O
from tests.helpers import cluster


def lj():
    return Table.analytic("lj", [1.0, 1.0], 0.1, 20.0)


def ang_model(radial=None):
    rad = radial or Table.analytic("exp_decay", [1.0, 1.0], 0.0, 20.0)
    return Model(FS_FAMILY_ANGULAR, 1, [lj(), rad, Table.analytic("harmonic", [1.0, -0.5], -1.0, 1.0)])


def triangle(r, x0=0.0):
    return cluster([[x0, 0, 0], [r, 0, 0], [r / 2.0, r * np.sqrt(3.0) / 2.0, 0]], 100.0)


def run(ds, model):
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model)
    return o.eval(1.0, 0.0)


def test_newton_third_law():
    out = run(triangle(2.5), ang_model())
    assert np.isfinite(out["energy"][0])
    assert np.linalg.norm(out["forces"].sum(axis=0)) <= 1e-11
    d = run(cluster([[0, 0, 0], [2.5, 0, 0]], 100.0), ang_model())
    assert np.linalg.norm(d["forces"].sum(axis=0)) <= 1e-12


def test_zero_radial_is_pair_only():
    zero = Table.analytic("const", [0.0], 0.0, 100.0)
    a = run(triangle(2.5), ang_model(zero))
    p = run(triangle(2.5), Model(FS_FAMILY_PAIR, 1, [lj()]))
    assert np.max(np.abs(a["forces"] - p["forces"])) <= 1e-12
    assert abs(a["energy"][0] - p["energy"][0]) <= 1e-12


def test_three_body_energy_and_fd_force():
    r = 2.5
    out = run(triangle(r), ang_model())
    # three angles of 60°: 3 · f(r)² · (cos 60° + ½)² on top of the pair sum
    lj_r = 4.0 * ((1 / r) ** 12 - (1 / r) ** 6)
    e3 = 3 * np.exp(-r) ** 2 * (0.5 + 0.5) ** 2
    assert abs(out["energy"][0] - (3 * lj_r + e3)) <= 1e-12 * abs(3 * lj_r + e3)
    dr = 1e-5
    ep = run(triangle(r, dr / 2), ang_model())["energy"][0]
    em = run(triangle(r, -dr / 2), ang_model())["energy"][0]
    fd = -(ep - em) / dr
    assert abs(out["forces"][0, 0] - fd) <= 1e-5 * abs(fd) + 1e-10
    again = run(triangle(r), ang_model())
    assert np.max(np.abs(again["forces"] - out["forces"])) <= 1e-14
    s = out["stress"][0].reshape(3, 3)
    assert np.max(np.abs(s - s.T)) <= 1e-13
