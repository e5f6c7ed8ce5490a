"""The oracle's Tersoff restatement, pinned against the reference's own unit
tests (tests/unit/test_tersoff_force.cpp): Si (1988) parameters, a dimer
and an equilateral triangle in a 100 Å box.

  DimerEnergyMatchesAnalytic      E = A e^{−λr} − B e^{−μr} at r = 2.35 (ζ = 0)   1e-10 rel
  DimerEnergyIsNegative / DimerNewtonThirdLaw                                     1e-11
  Dimer/TriangleForceConsistentWithEnergyFD   F_x(0) = −dE/dx₀, h = 1e-6 Å         1e-6 rel
  TriangleNewtonThirdLaw                                                          1e-10
  TriangleForcesIdempotent                                                        1e-14
  BeyondCutoffZeroContribution    r = 3.5 > S                                     1e-14
  StressSymmetric                                                                 1e-12
"""
import numpy as np

from forcesmith_b200.abi import FS_FAMILY_TERSOFF, Model, Table
from oracle import api as O
from tests.helpers import cluster

SI = dict(A=1830.8, B=471.18, lam=2.4799, mu=1.7322, beta=1.1e-6, n=0.78734, c=1.0039e5, d=16.217,
          h=-0.59825, R=2.7, S=3.0)


def si_model(**over):
    p = dict(SI, **over)
    return Model(FS_FAMILY_TERSOFF, 1, [Table.tersoff(**p)])


def dimer(r, x0=0.0):
    return cluster([[x0, 0, 0], [r, 0, 0]], 100.0)


def triangle(r, x0=0.0):
    return cluster([[x0, 0, 0], [r, 0, 0], [0.5 * r, r * np.sqrt(3.0) / 2.0, 0]], 100.0)


def run(ds, model=None):
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model or si_model())
    return o.eval(1.0, 0.0)


def test_dimer_energy_matches_analytic():
    r = 2.35
    out = run(dimer(r))
    e = SI["A"] * np.exp(-SI["lam"] * r) - SI["B"] * np.exp(-SI["mu"] * r)
    assert out["energy"][0] < 0.0
    assert abs(out["energy"][0] - e) <= 1e-10 * abs(e)
    assert np.linalg.norm(out["forces"].sum(axis=0)) <= 1e-11


def _fd_check(make, r):
    out = run(make(r))
    dr = 1e-6
    ep = run(make(r, dr / 2))["energy"][0]
    em = run(make(r, -dr / 2))["energy"][0]
    fd = -(ep - em) / dr
    fx = out["forces"][0, 0]
    assert abs(fx - fd) <= 1e-6 * abs(fd) + 1e-10, (fx, fd)
    return out


def test_dimer_force_consistent_with_energy_fd():
    _fd_check(dimer, 2.35)


def test_triangle_three_body():
    out = _fd_check(triangle, 2.4)
    assert np.linalg.norm(out["forces"].sum(axis=0)) <= 1e-10
    s = out["stress"][0].reshape(3, 3)
    assert np.max(np.abs(s - s.T)) <= 1e-12
    again = run(triangle(2.4))
    assert np.max(np.abs(again["forces"] - out["forces"])) <= 1e-14
    assert abs(again["energy"][0] - out["energy"][0]) <= 1e-14


def test_beyond_cutoff_zero():
    out = run(dimer(3.5))
    assert abs(out["energy"][0]) <= 1e-14
    assert np.max(np.abs(out["forces"])) <= 1e-14


def test_parameter_gather_order_and_bounds():
    """Gather order: the 12 fields per pair slot in declaration order, free
    ones only (tersoff_force.cpp:208-246); ω fixed by default."""
    m = Model(FS_FAMILY_TERSOFF, 2, [Table.tersoff(**dict(SI, A=SI["A"] * (1 + 0.01 * k))) for k in range(3)])
    o = O.Oracle()
    o.upload(cluster([[0, 0, 0], [2.3, 0, 0]], 20.0, types=[0, 1]))
    o.set_model(m)
    x = o.gather_params()
    assert x.size == 3 * 11
    assert np.allclose(x[::11], [SI["A"] * (1 + 0.01 * k) for k in range(3)])
    assert np.allclose(x[10::11], SI["S"])
