"""Shared builders for the parity tests: small datasets and models in the
shapes of the reference's unit-test fixtures and of the benchmark workloads."""
import numpy as np

from forcesmith_b200.abi import (Dataset, Model, Table, FS_FAMILY_ADP, FS_FAMILY_EAM,
                                 FS_FAMILY_PAIR, FS_FAMILY_SW)
from forcesmith_b200 import synth


def cluster(pos, box, types=None, ref_force=None):
    """A single periodic cubic configuration (make_cluster / make_binary of
    tests/unit/test_param_jacobian.cpp)."""
    pos = np.asarray(pos, np.float64).reshape(-1, 3)
    n = pos.shape[0]
    b = np.zeros(9)
    b[0] = b[4] = b[8] = box
    t = np.zeros(n, np.int32) if types is None else np.asarray(types, np.int32)
    return Dataset(np.array([n], np.int32), b.reshape(1, 9), pos, t,
                   np.zeros((n, 3)) if ref_force is None else np.asarray(ref_force, np.float64),
                   np.zeros(1), np.zeros((1, 9)))


def concat(*dss):
    dss = [d if d.ref_force is not None else with_zero_labels(d) for d in dss]
    return Dataset(np.concatenate([d.natoms for d in dss]).astype(np.int32),
                   np.concatenate([d.box9 for d in dss]),
                   np.concatenate([d.pos for d in dss]),
                   np.concatenate([d.type for d in dss]).astype(np.int32),
                   np.concatenate([d.ref_force for d in dss]),
                   np.concatenate([d.ref_energy for d in dss]),
                   np.concatenate([d.ref_stress9 for d in dss]))


def with_zero_labels(ds: Dataset) -> Dataset:
    return ds.with_labels(np.zeros((ds.n_atoms, 3)), np.zeros(ds.n_cfg), np.zeros((ds.n_cfg, 9)))


def label(ds: Dataset, model: Model, sess_factory, w_e=1.0, w_s=0.0):
    """Reference labels: the given model evaluated in FP64 by `sess_factory()`."""
    s = sess_factory()
    s.upload(with_zero_labels(ds))
    s.set_model(model)
    out = s.eval(w_e, w_s)
    return ds.with_labels(out["forces"], out["energy"], out["stress"])


def small_ternary(n_cfg=6, natoms=48, seed=99):
    return synth.packing(np.full(n_cfg, natoms, np.int32), seed=seed)


def ternary_models(nknots=20):
    true = synth.ternary_true_model(nknots)
    start = synth.perturb(true, 0.95, 1.05, seed=7)
    return true, start


def spline_pair_model(nt=2, nknots=12, rmin=1.5, rmax=5.5, seed=3):
    r = np.linspace(rmin, rmax, nknots)
    tabs = []
    k = 0
    for a in range(nt):
        for b in range(a, nt):
            f = synth.uniform(nknots, 0.9, 1.1, seed + k)
            k += 1
            y = 0.4 * (np.exp(-2.0 * (r - 2.6)) - 2.0 * np.exp(-(r - 2.6))) * f * (1 - (r / rmax) ** 4)
            tabs.append(Table.spline(rmin, rmax, y))
    return Model(FS_FAMILY_PAIR, nt, tabs)


def small_diamond(n_cfg=4, cells=(2,), seed=31):
    return synth.diamond(n_cfg, cells=cells, seed=seed)


def adp_spline_model(nt=2, nknots=10, seed=5):
    """Spline ADP tables: pair[np], density[nt], embedding[nt], dipole[np], quadrupole[np]."""
    r = np.linspace(1.8, 5.5, nknots)
    rho = np.linspace(0.0, 30.0, nknots)
    np_ = nt * (nt + 1) // 2
    tabs = []
    k = 0

    def f(lo, hi):
        nonlocal k
        k += 1
        return synth.uniform(nknots, lo, hi, seed + k)
    for _ in range(np_):
        tabs.append(Table.spline(1.8, 5.5, 0.3 * (np.exp(-2 * (r - 2.7)) - 2 * np.exp(-(r - 2.7))) * f(0.9, 1.1)
                                 * (1 - (r / 5.5) ** 4)))
    for _ in range(nt):
        tabs.append(Table.spline(1.8, 5.5, np.exp(-1.2 * (r - 2.5)) * f(0.9, 1.1) * (1 - (r / 5.5) ** 4)))
    for _ in range(nt):
        tabs.append(Table.spline(0.0, 30.0, -np.sqrt(rho) * f(0.9, 1.1)))
    for _ in range(np_):
        tabs.append(Table.spline(1.8, 5.5, 0.05 * np.exp(-(r - 2.5)) * f(0.5, 1.5) * (1 - (r / 5.5) ** 4)))
    for _ in range(np_):
        tabs.append(Table.spline(1.8, 5.5, 0.02 * np.exp(-1.5 * (r - 2.5)) * f(0.5, 1.5) * (1 - (r / 5.5) ** 4)))
    from forcesmith_b200.abi import FS_FAMILY_ADP
    return Model(FS_FAMILY_ADP, nt, tabs)
