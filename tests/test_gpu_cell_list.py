"""Device cell lists: neighbour sets bit-exact against the oracle's
brute-force build (the reference's build_periodic,
src/core/neighbor_list.cpp:59-92) on boxes where the cells prune.

The small cases of test_gpu_parity.py have at most two slabs per lattice
direction.  Here the boxes are cut into 3 to 8 slabs per direction, and the
cases cover:
  - large packings (1,500 and 2,000 atoms, rc = 6 Å),
  - diamond Si supercells at the Stillinger-Weber cutoff,
  - a strongly sheared triclinic box,
  - a slab box, narrow along one direction and wide along the others
    (one slab and two image shells along z, several slabs along x and y),
  - a configuration with an atom at fractional coordinate 0 and one just
    below 1 (cell edges),
  - several such configurations in one upload (cell offsets per configuration).
Bar: bit-exact counts, j and image codes, in the reference's order.
"""
import numpy as np
import pytest

from forcesmith_b200 import synth
from forcesmith_b200.abi import Dataset, Model, Table, FS_FAMILY_PAIR
from oracle import api as O
from tests.helpers import concat, with_zero_labels

pytestmark = pytest.mark.gpu


def _one(pos, box9, types=None):
    pos = np.asarray(pos, np.float64).reshape(-1, 3)
    n = pos.shape[0]
    t = np.zeros(n, np.int32) if types is None else np.asarray(types, np.int32)
    return with_zero_labels(Dataset(np.array([n], np.int32), np.asarray(box9, np.float64).reshape(1, 9), pos, t,
                                    None, None, None))


def _compare(ds, rcut):
    from forcesmith_b200.gpu import GpuSession
    model = Model(FS_FAMILY_PAIR, 1, [Table.spline(0.0, rcut, np.zeros(4))])
    ds.type[:] = 0
    g = GpuSession(0, "fp64")
    g.upload(ds)
    g.set_model(model)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model)
    assert g.num_pairs() == o.num_pairs()
    assert np.array_equal(g.neighbor_counts(ds.n_atoms), o.neighbor_counts(ds.n_atoms))
    gj, gimg = g.neighbors()
    oj, oimg, _ = o.neighbors()
    assert np.array_equal(gj, oj)
    assert np.array_equal(gimg, oimg)
    g.close()
    return int(o.num_pairs())


def test_cells_large_packings():
    ds = synth.packing(np.array([1500, 2000], np.int32), seed=41)
    assert _compare(ds, 6.0) > 0


def test_cells_diamond_supercells_sw_cutoff():
    ds = synth.diamond(n_cfg=3, cells=(4, 5), seed=17)
    assert _compare(ds, 1.80 * 2.0951) > 0


def test_cells_sheared_triclinic():
    rng = np.random.default_rng(7)
    a, b, c = 30.0, 28.0, 26.0
    box = np.array([[a, 0.45 * b, -0.3 * c], [0.0, b, 0.4 * c], [0.0, 0.0, c]])
    f = rng.uniform(0, 1, (900, 3))
    ds = _one(f @ box.T, box.reshape(9))
    assert _compare(ds, 5.0) > 0


def test_cells_slab_box():
    rng = np.random.default_rng(9)
    box = np.diag([40.0, 36.0, 2.5])
    f = rng.uniform(0, 1, (500, 3))
    ds = _one(f @ box.T, box.reshape(9))
    assert _compare(ds, 4.2) > 0


def test_cells_atoms_on_cell_edges():
    rng = np.random.default_rng(3)
    L = 24.0
    f = rng.uniform(0, 1, (300, 3))
    f[0] = [0.0, 0.0, 0.0]
    f[1] = [np.nextafter(1.0, 0.0), 0.5, np.nextafter(1.0, 0.0)]
    f[2] = [1.0 / 3.0, 2.0 / 3.0, 0.25]
    f[3] = [0.5, 0.5, 0.5]
    ds = _one(f * L, np.diag([L, L, L]).reshape(9))
    assert _compare(ds, 6.0) > 0


def test_cells_mixed_upload():
    rng = np.random.default_rng(5)
    parts = [synth.packing(np.array([64, 700], np.int32), seed=12)]
    box = np.array([[20.0, 6.0, 0.0], [0.0, 19.0, 3.0], [0.0, 0.0, 21.0]])
    parts.append(_one(rng.uniform(0, 1, (400, 3)) @ box.T, box.reshape(9)))
    parts.append(synth.diamond(n_cfg=1, cells=(2,), seed=4))
    ds = concat(*parts)
    assert _compare(ds, 6.0) > 0
