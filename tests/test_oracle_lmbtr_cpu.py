"""The oracle's LMBTR + linear-head restatement, pinned against the
reference's unit tests (tests/unit/test_lmbtr.cpp): the 4-atom environment
(origin plus three neighbours) in a 100 Å box, rcut = 6, weight_scale = 3,
k2 grid (0, 6, 6 bins, σ 0.4), k3 grid (−1, 1, 6 bins, σ 0.2).

  DescriptorSizeFormula    S·n2 + P·n3, either term absent
  K3OnlyMatchesTail        k3-only descriptor = the k3 tail of both      1e-14
  L2Normalized             ‖D‖ = 1                                        1e-12
  Translation / Rotation / PermutationInvariant                          1e-10 / 1e-9 / 1e-12
  SensitiveToGeometry      moving a neighbour changes D by > 1e-3
  ForceMatchesEnergyFD     forces (central-difference descriptor gradient)
                           against −ΔE/Δx, Δx = 1e-5                   1e-4·|fd| + 1e-5
plus a dimer's k2 bins by hand (Gaussian of r, weight e^{−r/3}) and
Newton's third law.
"""
import numpy as np

from forcesmith_b200.abi import FS_FAMILY_LMBTR, Model, Table, lmbtr_size
from oracle import api as O
from tests.helpers import cluster

ENV = np.array([[0.0, 0.0, 0.0], [2.1, 0.3, -0.2], [0.4, 2.0, 0.5], [-1.3, 0.7, 1.9]])
K2 = (0.0, 6.0, 6, 0.4)
K3 = (-1.0, 1.0, 6, 0.2)


def spec(k2=K2, k3=K3, normalize=True):
    return Table.lmbtr(6.0, 3.0, normalize, k2, k3)


def oracle(pos, sp, coeffs=None, nt=1, types=None):
    S = lmbtr_size(sp, nt)
    w = np.zeros(S) if coeffs is None else coeffs
    o = O.Oracle()
    o.upload(cluster(pos, 100.0, types=types))
    o.set_model(Model(FS_FAMILY_LMBTR, nt, [sp] + [Table.linear_head(w, 0.0) for _ in range(nt)]))
    return o, S


def desc(pos, sp, i=0):
    o, S = oracle(pos, sp)
    return o.descriptor(0, i, S)


def test_descriptor_size_formula():
    for S in (1, 2):
        P = S * (S + 1) // 2
        assert lmbtr_size(spec(), S) == S * 6 + P * 6
        assert lmbtr_size(spec(k3=None), S) == S * 6
        assert lmbtr_size(spec(k2=None), S) == P * 6


def test_k3_only_matches_tail():
    both = desc(ENV, spec(normalize=False))
    k3 = desc(ENV, spec(k2=None, normalize=False))
    assert k3.size == both.size - 6
    assert np.linalg.norm(k3 - both[6:]) <= 1e-14
    assert np.linalg.norm(k3) > 1e-6


def test_l2_normalized():
    assert abs(np.linalg.norm(desc(ENV, spec())) - 1.0) <= 1e-12


def test_invariances():
    v0 = desc(ENV, spec())
    assert np.linalg.norm(desc(ENV + np.array([3.7, -1.2, 0.9]), spec()) - v0) <= 1e-10
    ax = np.array([0.3, -0.8, 0.5])
    ax /= np.linalg.norm(ax)
    th = 0.7
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    R = np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K
    assert np.linalg.norm(desc(ENV @ R.T, spec()) - v0) <= 1e-9
    perm = ENV[[0, 3, 2, 1]]
    assert np.linalg.norm(desc(perm, spec()) - v0) <= 1e-12


def test_sensitive_to_geometry():
    v0 = desc(ENV, spec(normalize=False))
    moved = ENV.copy()
    moved[1] += [0.4, -0.3, 0.2]
    assert np.linalg.norm(desc(moved, spec(normalize=False)) - v0) > 1e-3


def test_dimer_k2_bins_by_hand():
    r = 2.3
    v = desc([[0, 0, 0], [r, 0, 0]], spec(k3=None, normalize=False))
    lo, hi, n, sig = K2
    x = np.linspace(lo, hi, n)
    g = np.exp(-r / 3.0) / (sig * np.sqrt(2 * np.pi)) * np.exp(-(x - r) ** 2 / (2 * sig * sig))
    g[np.abs(x - r) > 5 * sig] = 0.0  # outside the 5σ window
    assert np.abs(v - g).max() <= 1e-14 * np.abs(g).max() * 10


def test_force_matches_energy_fd_and_newton():
    S = lmbtr_size(spec(), 1)
    w = 0.1 + 0.03 * np.arange(S)
    o, _ = oracle(ENV, spec(), w)
    out = o.eval(1.0, 0.0)
    F = out["forces"].reshape(-1, 3)
    assert np.abs(F.sum(axis=0)).max() <= 1e-10 * np.abs(F).max()

    def energy(pos):
        oo, _ = oracle(pos, spec(), w)
        return oo.eval(1.0, 0.0)["energy"][0]

    dr = 1e-5
    for a in range(4):
        for c in range(3):
            p, m = ENV.copy(), ENV.copy()
            p[a, c] += dr / 2
            m[a, c] -= dr / 2
            fd = -(energy(p) - energy(m)) / dr
            assert abs(F[a, c] - fd) <= 1e-4 * abs(fd) + 1e-5, (a, c)


# ---- the model JSON (force_model_reader.cpp:350-382, output_writer.cpp:238-267)

def test_reader_round_trip_case():
    """The reference's Lmbtr.ReaderRoundTrip input: 8-bin k2 and k3 grids,
    one species, so S = 16."""
    import json
    from forcesmith_b200 import io
    text = json.dumps({
        "model": "ml", "ntypes": 1,
        "descriptor": {"type": "lmbtr", "rcut": 6.0, "weight_scale": 3.0, "normalize": True,
                       "k2": {"min": 0.0, "max": 6.0, "n": 8, "sigma": 0.3},
                       "k3": {"min": -1.0, "max": 1.0, "n": 8, "sigma": 0.1}},
        "heads": [{"type": "linear", "coeffs": [0] * 16, "bias": 0.0}]})
    m = io.read_model(text)
    assert m.family == FS_FAMILY_LMBTR and lmbtr_size(m.tables[0], 1) == 16
    v = m.tables[0].values
    assert int(v[3]) == 8 and int(v[7]) == 8
    m2 = io.read_model(io.write_model(m))
    assert np.array_equal(m2.tables[0].values, v)
    assert np.array_equal(m2.tables[1].values, m.tables[1].values)


def test_reader_defaults_and_errors():
    import json
    import pytest
    from forcesmith_b200 import io

    def read(desc, nt=1, S=None):
        sp = io._read_lmbtr(desc)
        S = lmbtr_size(sp, nt) if S is None else S
        return io.read_model(json.dumps({"model": "ml", "ntypes": nt, "descriptor": desc,
                                         "heads": [{"coeffs": [0.0] * S} for _ in range(nt)]}))

    m = read({"type": "lmbtr", "rcut": 5.0})
    v = m.tables[0].values
    # weight_scale = rcut / 2; both grids at their defaults, k2 up to rcut
    assert v[1] == 2.5 and v[2] == 1.0 and list(v[3:7]) == [50, 0.0, 5.0, 0.3] and list(v[7:]) == [50, -1.0, 1.0, 0.1]
    m = read({"type": "lmbtr", "k3": {"n": 12}}, nt=2)  # naming k3 drops k2
    v = m.tables[0].values
    assert v[3] == 0 and v[7] == 12 and lmbtr_size(m.tables[0], 2) == 36
    with pytest.raises(io.FormatError):
        io._read_lmbtr({"type": "lmbtr", "k2": {"n": 0}})
    with pytest.raises(io.FormatError):  # head length must match S
        io.read_model(json.dumps({"model": "ml", "ntypes": 1, "descriptor": {"type": "lmbtr"},
                                  "heads": [{"coeffs": [0.0] * 5}]}))


def test_standardization_block_round_trip():
    from forcesmith_b200 import io
    sp = spec()
    S = lmbtr_size(sp, 2)
    rng = np.random.default_rng(4)
    m = Model(FS_FAMILY_LMBTR, 2, [sp] + [Table.linear_head(rng.normal(size=S), 0.5) for _ in range(2)])
    m = m.with_standardization(rng.normal(size=(2, S)), rng.uniform(0.5, 2, (2, S)))
    m2 = io.read_model(io.write_model(m))
    assert len(m2.tables) == 5
    for a, b in zip(m.tables, m2.tables):
        assert np.array_equal(a.values, b.values)


def test_model_validation():
    """Malformed LMBTR tables and heads of the wrong length are refused."""
    import pytest
    from forcesmith_b200.abi import FsError
    o = O.Oracle()
    o.upload(cluster(ENV, 100.0))
    good = spec()
    S = lmbtr_size(good, 1)
    o.set_model(Model(FS_FAMILY_LMBTR, 1, [good, Table.linear_head(np.zeros(S))]))
    bad = []
    for k, v in ((0, 0.0), (1, -1.0), (3, 2.5), (6, 0.0)):  # rcut, weight scale, fractional n, sigma
        t = spec()
        t.values[k] = v
        bad.append(Model(FS_FAMILY_LMBTR, 1, [t, Table.linear_head(np.zeros(S))]))
    t = spec()
    t.values[3] = t.values[7] = 0  # no term
    bad.append(Model(FS_FAMILY_LMBTR, 1, [t, Table.linear_head(np.zeros(1))]))
    bad.append(Model(FS_FAMILY_LMBTR, 1, [good, Table.linear_head(np.zeros(S + 1))]))
    for m in bad:
        with pytest.raises(FsError):
            o.set_model(m)


def test_two_species_block_layout():
    """LmbtrLayout (lmbtr.hpp:13-38, DescriptorLayout::index = base + chan ·
    count + t): k2 blocks per neighbour species, then k3 blocks per species
    pair in pair_ordinal order.  A species-0 atom with one species-0 and one
    species-1 neighbour fills the k2 blocks of both species and only the k3
    block of the pair (0, 1), ordinal 1 of {(0,0), (0,1), (1,1)}."""
    sp = spec(normalize=False)
    o = O.Oracle()
    o.upload(cluster([[0, 0, 0], [2.2, 0.3, 0.0], [-0.5, 2.1, 0.4]], 100.0, types=[0, 0, 1]))
    o.set_model(Model(FS_FAMILY_LMBTR, 2, [sp] + [Table.linear_head(np.zeros(lmbtr_size(sp, 2)))] * 2))
    v = o.descriptor(0, 0, lmbtr_size(sp, 2))
    n2, n3 = 6, 6
    k2 = v[:2 * n2].reshape(2, n2)
    k3 = v[2 * n2:].reshape(3, n3)
    assert np.abs(k2[0]).max() > 0 and np.abs(k2[1]).max() > 0
    assert np.abs(k3[1]).max() > 0 and np.abs(k3[0]).max() == 0 and np.abs(k3[2]).max() == 0
    # species-0 block of k2 is the species-0 neighbour's Gaussian alone
    r = np.linalg.norm([2.2, 0.3, 0.0])
    x = np.linspace(0.0, 6.0, n2)
    g = np.exp(-r / 3.0) / (0.4 * np.sqrt(2 * np.pi)) * np.exp(-(x - r) ** 2 / (2 * 0.4 ** 2))
    g[np.abs(x - r) > 5 * 0.4] = 0.0
    assert np.abs(k2[0] - g).max() <= 1e-14
