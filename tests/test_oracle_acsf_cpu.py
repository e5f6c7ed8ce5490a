"""The oracle's ACSF + linear-head restatement, pinned against the
reference's unit tests (tests/unit/test_acsf.cpp, tests/unit/test_ml_force.cpp):
the 4-atom environment (origin plus three neighbours) and the dimer in a
100 Å box, rcut = 6.

  DescriptorSizeFormula    S = nt(1 + 2 + 1) + npair(2 + 1)
  G1HandValue / G3HandValue / DimerDescriptorMatchesHand
                           energies of a unit head = Σ_i D_i, by hand       1e-12
  AnalyticForceMatchesEnergyFD, NewtonThirdLaw, BeyondCutoffZero
"""
import numpy as np
import pytest

from forcesmith_b200.abi import FS_FAMILY_ACSF, Model, Table, acsf_size
from oracle import api as O
from tests.helpers import cluster

ENV = [[0.0, 0.0, 0.0], [2.1, 0.3, -0.2], [0.4, 2.0, 0.5], [-1.3, 0.7, 1.9]]


def fc(r, rc=6.0):
    return np.where(r < rc, 0.5 * (1 + np.cos(np.pi * r / rc)), 0.0)


def run(pos, spec, coeffs, bias=0.0, types=None, nt=1):
    heads = [Table.linear_head(coeffs, bias) for _ in range(nt)]
    o = O.Oracle()
    o.upload(cluster(pos, 100.0, types=types))
    o.set_model(Model(FS_FAMILY_ACSF, nt, [spec] + heads))
    return o.eval(1.0, 0.0)


def pair_dists(pos):
    p = np.asarray(pos)
    d = np.linalg.norm(p[:, None] - p[None], axis=-1)
    return d[~np.eye(len(p), dtype=bool)]


def test_descriptor_size_formula():
    spec = Table.acsf(6.0, g1=1, g2=[(1.0, 0.0), (0.5, 1.0)], g3=[1.0], g4=[(1.0, 1.0, 1.0), (0.5, 2.0, -1.0)],
                      g5=[(1.0, 1.0, 1.0)])
    for S in (1, 2, 3):
        assert acsf_size(spec, S) == S * (1 + 2 + 1) + S * (S + 1) // 2 * (2 + 1)


def test_g1_g3_hand_values():
    r = pair_dists(ENV)
    out = run(ENV, Table.acsf(6.0, g1=1), [1.0])
    assert abs(out["energy"][0] - fc(r).sum()) <= 1e-12
    out = run(ENV, Table.acsf(6.0, g3=[1.3]), [1.0])
    assert abs(out["energy"][0] - (np.cos(1.3 * r) * fc(r)).sum()) <= 1e-12


def test_dimer_g2_hand_value_and_bias():
    r, eta, rs = 2.5, 0.8, 1.0
    out = run([[0, 0, 0], [r, 0, 0]], Table.acsf(6.0, g2=[(eta, rs)]), [1.0], bias=0.25)
    e = np.exp(-eta * (r - rs) ** 2) * fc(np.array(r))
    assert abs(out["energy"][0] - 2 * (e + 0.25)) <= 1e-12


@pytest.mark.parametrize("angular", [False, True])
def test_forces_match_energy_fd_and_newton(angular):
    spec = Table.acsf(6.0, g1=1, g2=[(0.5, 0.0), (1.2, 1.5)], g3=[0.9],
                      g4=[(0.3, 1.0, 1.0), (0.2, 2.0, -1.0)] if angular else (),
                      g5=[(0.4, 1.5, 1.0)] if angular else ())
    w = np.linspace(0.3, -0.2, acsf_size(spec, 1))
    out = run(ENV, spec, w)
    assert np.linalg.norm(out["forces"].sum(axis=0)) <= 1e-12
    h = 1e-6
    for atom in (0, 2):
        for a in range(3):
            pp = np.array(ENV, float)
            pp[atom, a] += h
            pm = np.array(ENV, float)
            pm[atom, a] -= h
            fd = -(run(pp, spec, w)["energy"][0] - run(pm, spec, w)["energy"][0]) / (2 * h)
            assert abs(out["forces"][atom, a] - fd) <= 1e-6 * abs(fd) + 1e-9, (atom, a)
    s = out["stress"][0].reshape(3, 3)
    assert np.max(np.abs(s - s.T)) <= 1e-12


def test_beyond_cutoff_zero_and_species_channels():
    out = run([[0, 0, 0], [6.5, 0, 0]], Table.acsf(6.0, g2=[(0.5, 0.0)]), [1.0])
    assert abs(out["energy"][0]) <= 1e-14 and np.max(np.abs(out["forces"])) <= 1e-14
    # two species, every atom of species 0: the species-1 channel stays empty,
    # so its coefficient changes nothing
    spec = Table.acsf(6.0, g2=[(0.5, 0.0)])
    a = run(ENV, spec, [1.0, 0.0], nt=2, types=[0, 0, 0, 0])
    b = run(ENV, spec, [1.0, 5.0], nt=2, types=[0, 0, 0, 0])
    assert abs(a["energy"][0] - b["energy"][0]) <= 1e-14


# ---- feature standardization (MLBase::compute_standardization and
# standardize_in_place, ml_force.hpp:607-688), on the environment of the
# reference's ML_Standardization_RoundTrips test (test_force_model_reader.cpp)
STD_G2 = [(0.5, 0.0), (1.2, 1.5), (0.3, 2.5)]


def _hand_descriptors(pos, g2, rc=6.0):
    p = np.asarray(pos, np.float64)
    D = np.zeros((len(p), len(g2)))
    for i in range(len(p)):
        r = np.linalg.norm(np.delete(p, i, 0) - p[i], axis=1)
        for k, (eta, rs) in enumerate(g2):
            D[i, k] = np.sum(np.exp(-eta * (r - rs) ** 2) * fc(r, rc))
    return D


def _std_model(w, b, mean, inv_std):
    spec = Table.acsf(6.0, g2=STD_G2)
    return Model(FS_FAMILY_ACSF, 1, [spec, Table.linear_head(w, b)]).with_standardization([mean], [inv_std])


def test_standardization_statistics_and_energy():
    """mean and 1/σ per descriptor over the four atoms against numpy on hand
    descriptors (1e-12); the standardized head's energy
    Σ_i b + w·(D_i − mean) ⊙ inv_std by hand (1e-12)."""
    spec = Table.acsf(6.0, g2=STD_G2)
    w, b = np.array([0.7, -0.4, 0.25]), 0.1
    o = O.Oracle()
    o.upload(cluster(ENV, 100.0))
    o.set_model(Model(FS_FAMILY_ACSF, 1, [spec, Table.linear_head(w, b)]))
    mean, inv_std, count = o.acsf_standardization()
    D = _hand_descriptors(ENV, STD_G2)
    mu, var = D.mean(axis=0), (D ** 2).mean(axis=0) - D.mean(axis=0) ** 2
    assert count.tolist() == [4]
    np.testing.assert_allclose(mean[0], mu, rtol=1e-12, atol=0)
    np.testing.assert_allclose(inv_std[0], 1.0 / np.sqrt(var), rtol=1e-10, atol=0)
    o.set_model(_std_model(w, b, mean[0], inv_std[0]))
    e = o.eval(1.0, 0.0)["energy"][0]
    e_hand = np.sum(b + ((D - mean[0]) * inv_std[0]) @ w)
    assert abs(e - e_hand) <= 1e-12 * (1 + abs(e_hand))


def test_standardized_forces_match_energy_fd():
    """Forces of the standardized model against central differences of its
    energy (h = 1e-6, |Δ| ≤ 1e-7), and the same forces and energy as the
    unstandardized head w ⊙ inv_std, b − Σ w·inv_std·mean (1e-13, 1e-12)."""
    w, b = np.array([0.7, -0.4, 0.25]), 0.1
    mean, inv_std = np.array([0.3, 0.6, 0.9]), np.array([1.7, 0.8, 2.2])
    m = _std_model(w, b, mean, inv_std)
    o = O.Oracle()
    o.upload(cluster(ENV, 100.0))
    o.set_model(m)
    out = o.eval(1.0, 0.0)
    weff, beff = w * inv_std, b - np.sum(w * inv_std * mean)
    h = 1e-6
    for a in range(4):
        for x in range(3):
            pp, pm = np.array(ENV, float), np.array(ENV, float)
            pp[a, x] += h
            pm[a, x] -= h
            ep = run(pp, Table.acsf(6.0, g2=STD_G2), weff, beff)["energy"][0]
            em = run(pm, Table.acsf(6.0, g2=STD_G2), weff, beff)["energy"][0]
            assert abs(out["forces"][a][x] + (ep - em) / (2 * h)) <= 1e-7
    raw = run(ENV, Table.acsf(6.0, g2=STD_G2), weff, beff)
    np.testing.assert_allclose(out["forces"], raw["forces"], rtol=0, atol=1e-13)
    assert abs(out["energy"][0] - raw["energy"][0]) <= 1e-12


def test_standardization_tables_are_fixed():
    """A standardization value marked free is rejected by set_model."""
    from forcesmith_b200.abi import FsError
    m = _std_model([0.7, -0.4, 0.25], 0.1, [0.3, 0.6, 0.9], [1.7, 0.8, 2.2])
    m.tables[-1].fixed[0] = 0
    o = O.Oracle()
    o.upload(cluster(ENV, 100.0))
    with pytest.raises(FsError):
        o.set_model(m)


# ---- species re-ranking (MLBase::remap, ml_force.hpp:165-190; remap_layout,
# descriptor_layout.cpp:9-50)
REMAP_SPEC = Table.acsf(6.0, g1=1, g2=[(0.5, 1.0)], g3=[1.1], g4=[(0.1, 2.0, -1.0)], g5=[(0.2, 1.0, 1.0)])


def _two_species_model(seed=4):
    S = acsf_size(REMAP_SPEC, 2)
    rng = np.random.default_rng(seed)
    return Model(FS_FAMILY_ACSF, 2, [REMAP_SPEC] + [Table.linear_head(rng.normal(0, 0.3, S), -1.0 + t)
                                                   for t in range(2)])


def _eval(model, types, nt):
    o = O.Oracle()
    o.upload(cluster(ENV, 100.0, types=types))
    o.set_model(model)
    return o.eval(1.0, 0.0)


def test_remap_swapped_species_is_a_relabelling():
    """Remapping [A, B] → [B, A] and swapping every atom's species leaves the
    energy and forces unchanged (1e-12): each coefficient moves with its
    species channel, pair channels included."""
    m = _two_species_model()
    types = np.array([0, 1, 0, 1])
    ref = _eval(m, types, 2)
    r = m.acsf_remapped(["A", "B"], ["B", "A"])
    out = _eval(r, 1 - types, 2)
    assert abs(out["energy"][0] - ref["energy"][0]) <= 1e-12 * (1 + abs(ref["energy"][0]))
    np.testing.assert_allclose(out["forces"], ref["forces"], rtol=0, atol=1e-12)


def test_remap_added_species_changes_nothing():
    """Remapping [A, B] → [A, B, C]: with no atom of species C, energies and
    forces are those of the two-species model (1e-12); C's head is a zero
    head with free coefficients and a fixed zero bias, and the channels that
    involve C have coefficient 0."""
    m = _two_species_model()
    types = np.array([0, 1, 1, 0])
    ref = _eval(m, types, 2)
    r = m.acsf_remapped(["A", "B"], ["A", "B", "C"])
    assert r.ntypes == 3 and len(r.tables) == 4
    S3 = acsf_size(REMAP_SPEC, 3)
    assert r.tables[3].values.tolist() == [0.0] * (S3 + 1)
    assert r.tables[3].fixed[:-1].tolist() == [0] * S3 and r.tables[3].fixed[-1] == 1
    out = _eval(r, types, 3)
    assert abs(out["energy"][0] - ref["energy"][0]) <= 1e-12 * (1 + abs(ref["energy"][0]))
    np.testing.assert_allclose(out["forces"], ref["forces"], rtol=0, atol=1e-12)


def test_remap_drops_standardization():
    """remap clears the (old-layout) standardization."""
    m = _two_species_model()
    S = acsf_size(REMAP_SPEC, 2)
    ms = m.with_standardization(np.zeros((2, S)), np.ones((2, S)))
    assert len(ms.acsf_remapped(["A", "B"], ["B", "A"]).tables) == 3


def test_standardization_dead_features():
    """A feature with no variance across the atoms (both atoms of a dimer see
    the same environment) gets inv_std 0 (var ≤ 1e-12,
    compute_standardization) and drops out of the head: the standardized
    energy is N·b and the forces vanish (1e-12)."""
    spec = Table.acsf(6.0, g2=STD_G2)
    w, b = np.array([0.7, -0.4, 0.25]), 0.1
    dimer = [[0.0, 0.0, 0.0], [2.3, 0.0, 0.0]]
    o = O.Oracle()
    o.upload(cluster(dimer, 100.0))
    o.set_model(Model(FS_FAMILY_ACSF, 1, [spec, Table.linear_head(w, b)]))
    mean, inv_std, count = o.acsf_standardization()
    assert count.tolist() == [2] and np.all(inv_std == 0.0) and np.all(mean > 0)
    o.set_model(_std_model(w, b, mean[0], inv_std[0]))
    out = o.eval(1.0, 0.0)
    assert abs(out["energy"][0] - 2 * b) <= 1e-12
    assert np.max(np.abs(out["forces"])) <= 1e-12
