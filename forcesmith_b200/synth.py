"""Seeded synthetic workloads with the benchmark shapes.

No public dataset is involved: the workloads are generated here with fixed
seeds, and reference labels come from evaluating a seeded "true" model in
FP64.  Shapes:

  fcc_al        20 × fcc Al 3×3×3 (108 atoms), a = 4.05 Å, isotropic strain
                U[0.97, 1.03], Gaussian displacement σ = 0.10 Å.
  ternary       500 × 256 atoms, random sequential packing (d_min 2.2 Å,
                0.060 Å⁻³), 5 % random symmetric strain, species i.i.d.
                Zr 0.5 / Cu 0.4 / Al 0.1 in Z-sorted slots Al=0, Cu=1, Zr=2.
                Model: 6 φ + 3 ρ + 3 F makima splines × 20 knots (D = 240),
                cutoff 6.0 Å.
  sw_si         1000 diamond-Si configs of 2³/3³/4³ cells (64/216/512 atoms),
                a = 5.431 Å, σ = 0.15 Å, volumetric strain U[0.95, 1.05].
  de_ternary    200 × U{32…512} atoms of the ternary packing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build
from .abi import Dataset, Model, Table, FS_FAMILY_EAM, FS_FAMILY_SW, _dp, _ip

_SYN = None


def _lib():
    global _SYN
    if _SYN is None:
        _SYN = C.CDLL(_build.build_synth())
        L = _SYN
        L.fs_synth_fcc.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_uint64, C.POINTER(C.c_int32),
                                   C.POINTER(C.c_double), C.POINTER(C.c_double),
                                   C.POINTER(C.c_int32)]
        L.fs_synth_diamond.argtypes = [C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_uint64,
                                       C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double), C.POINTER(C.c_int32), C.c_int64]
        L.fs_synth_packing.argtypes = [C.c_int32, C.POINTER(C.c_int32), C.c_double, C.c_double,
                                       C.c_double, C.POINTER(C.c_double), C.c_int32, C.c_uint64,
                                       C.POINTER(C.c_double), C.POINTER(C.c_double),
                                       C.POINTER(C.c_int32)]
        L.fs_synth_counts.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_uint64,
                                      C.POINTER(C.c_int32)]
        L.fs_synth_uniform.argtypes = [C.c_int64, C.c_double, C.c_double, C.c_uint64,
                                       C.POINTER(C.c_double)]
    return _SYN


def uniform(n, lo, hi, seed):
    out = np.zeros(int(n))
    _lib().fs_synth_uniform(int(n), lo, hi, seed, _dp(out))
    return out


def fcc(n_cfg=20, ncell=3, a=4.05, sigma=0.10, s_lo=0.97, s_hi=1.03, seed=20261203):
    n = 4 * ncell ** 3
    natoms = np.zeros(n_cfg, np.int32)
    box = np.zeros((n_cfg, 9))
    pos = np.zeros((n_cfg * n, 3))
    typ = np.zeros(n_cfg * n, np.int32)
    _lib().fs_synth_fcc(n_cfg, ncell, a, sigma, s_lo, s_hi, seed, _ip(natoms), _dp(box), _dp(pos),
                        _ip(typ))
    return Dataset(natoms, box, pos, typ)


def diamond(n_cfg=1000, cells=(2, 3, 4), a=5.431, sigma=0.15, v_lo=0.95, v_hi=1.05,
            seed=20261205):
    ch = np.array(cells, np.int32)
    cap = n_cfg * 8 * int(max(cells)) ** 3
    natoms = np.zeros(n_cfg, np.int32)
    box = np.zeros((n_cfg, 9))
    pos = np.zeros((cap, 3))
    typ = np.zeros(cap, np.int32)
    rc = _lib().fs_synth_diamond(n_cfg, _ip(ch), ch.size, a, sigma, v_lo, v_hi, seed, _ip(natoms),
                                 _dp(box), _dp(pos), _ip(typ), cap)
    assert rc == 0
    N = int(natoms.sum())
    return Dataset(natoms, box, np.ascontiguousarray(pos[:N]), np.ascontiguousarray(typ[:N]))


TERNARY_PROB = (0.1, 0.4, 0.5)  # Al, Cu, Zr (Z-sorted slots)


def packing(natoms, density=0.060, dmin=2.2, strain=0.05, prob=TERNARY_PROB, seed=20261204):
    natoms = np.ascontiguousarray(natoms, np.int32)
    N = int(natoms.sum())
    box = np.zeros((natoms.size, 9))
    pos = np.zeros((N, 3))
    typ = np.zeros(N, np.int32)
    p = np.ascontiguousarray(prob, np.float64)
    rc = _lib().fs_synth_packing(natoms.size, _ip(natoms), density, dmin, strain, _dp(p), p.size,
                                 seed, _dp(box), _dp(pos), _ip(typ))
    if rc != 0:
        raise RuntimeError(f"packing failed for config {-rc - 1}")
    return Dataset(natoms, box, pos, typ)


def ternary_geometry(n_cfg=500, natoms=256, seed=20261204):
    return packing(np.full(n_cfg, natoms, np.int32), seed=seed)


def de_geometry(n_cfg=200, lo=32, hi=512, seed=20261206):
    counts = np.zeros(n_cfg, np.int32)
    _lib().fs_synth_counts(n_cfg, lo, hi, seed, _ip(counts))
    return packing(counts, seed=seed + 1)


# ---------------------------------------------------------------------------
# Models
# ---------------------------------------------------------------------------

RC_TERNARY = 6.0
R_LO = 1.8
RHO_MAX = 24.0  # embedding domain [0, RHO_MAX]; chosen above every ρ_i of the workloads


def _taper(r, lo, hi):
    return 1.0 - ((r - lo) / (hi - lo)) ** 6


def ternary_true_model(nknots=20):
    """6 φ + 3 ρ + 3 F makima splines on uniform grids (slots Al, Cu, Zr)."""
    nt = 3
    r = np.linspace(R_LO, RC_TERNARY, nknots)
    r0 = np.array([2.86, 2.55, 3.20])        # Al, Cu, Zr nearest-neighbour distances
    De = np.array([0.28, 0.33, 0.42])
    alpha = 1.55
    tables = []
    for a in range(nt):
        for b in range(a, nt):
            rr = 0.5 * (r0[a] + r0[b])
            D = np.sqrt(De[a] * De[b])
            e = np.exp(-alpha * (r - rr))
            tables.append(Table.spline(R_LO, RC_TERNARY, D * (e * e - 2 * e) * _taper(r, R_LO, RC_TERNARY)))
    A = np.array([1.00, 1.20, 0.90])
    beta = np.array([1.25, 1.35, 1.10])
    for a in range(nt):
        tables.append(Table.spline(R_LO, RC_TERNARY,
                                   A[a] * np.exp(-beta[a] * (r - 2.5)) * _taper(r, R_LO, RC_TERNARY)))
    rho = np.linspace(0.0, RHO_MAX, nknots)
    E = np.array([1.30, 1.55, 1.95])
    c2 = np.array([0.010, 0.012, 0.008])
    for a in range(nt):
        tables.append(Table.spline(0.0, RHO_MAX, -E[a] * np.sqrt(rho) + c2[a] * rho ** 2))
    return Model(FS_FAMILY_EAM, nt, tables)


def perturb(model: Model, lo=0.95, hi=1.05, seed=7):
    """Multiplies every free value by U[lo, hi] (the start model of a fit)."""
    x = model.free_values()
    f = uniform(x.size, lo, hi, seed)
    return model.with_values(x * f)


# Stillinger–Weber Si (textbook ε, σ, a, λ, γ, A, B) mapped to the
# reference's parameterisation (tests/unit/test_stiweb_force.cpp:27-38).
SW_TEXTBOOK = dict(eps=2.1683, sigma=2.0951, a=1.80, lam=21.0, gamma=1.20,
                   A=7.049556277, B=0.6022245584)


def sw_model(eps=2.1683, sigma=2.0951, a=1.80, lam=21.0, gamma=1.20, A=7.049556277,
             B=0.6022245584, p=4.0, q=0.0):
    fixed = np.array([0, 0, 1, 1, 0, 0, 0, 0], np.uint8)  # p, q fixed
    t = Table.sw(A * eps * B * sigma ** p, A * eps * sigma ** q, p, q, sigma, a * sigma,
                 gamma * sigma, a * sigma, fixed=fixed)
    return Model(FS_FAMILY_SW, 1, [t, Table.lam([lam * eps])])


def sw_start_model(seed=11, frac=0.10):
    f = uniform(7, 1.0 - frac, 1.0 + frac, seed)
    kw = dict(SW_TEXTBOOK)
    for k, key in enumerate(("eps", "sigma", "a", "lam", "gamma", "A", "B")):
        kw[key] = kw[key] * f[k]
    return sw_model(**kw)
