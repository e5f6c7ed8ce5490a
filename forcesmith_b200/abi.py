"""ctypes mirror of include/forcesmith_gpu.h and a thin session wrapper.

The same `Session` class drives any library that exports the `fs_gpu_*`
call set under some prefix, so host code (and the parity tests) read the
same for the device library and for any CPU implementation of the ABI.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

FS_OK = 0
FS_ERR_ARG = -1
FS_ERR_CUDA = -2
FS_ERR_STATE = -3
FS_ERR_UNSUPPORTED = -4
FS_ERR_NOMEM = -5
FS_ERR_DEVICE = -6
FS_ERR_NUMERIC = -7

FS_FAMILY_PAIR, FS_FAMILY_EAM, FS_FAMILY_ADP, FS_FAMILY_SW, FS_FAMILY_TERSOFF, FS_FAMILY_ANGULAR = 0, 1, 2, 3, 4, 5
FS_FAMILY_ACSF = 6
FS_FAMILY_LMBTR = 7
FS_TABLE_SPLINE, FS_TABLE_ANALYTIC, FS_TABLE_SW, FS_TABLE_LAMBDA, FS_TABLE_TERSOFF = 0, 1, 2, 3, 4
FS_TABLE_ACSF, FS_TABLE_LINEAR_HEAD, FS_TABLE_STANDARDIZATION = 5, 6, 7
FS_TABLE_LMBTR = 8
TERSOFF_FIELDS = ("A", "B", "lambda", "mu", "beta", "n", "c", "d", "h", "R", "S", "omega")
FS_PREC_FP32, FS_PREC_FP64 = 0, 1

FORMS = {  # name: (fs_form id, parameter count), analytic_potential.hpp:801-806
    "lj": (0, 2), "morse": (1, 3), "exp_decay": (2, 2), "sqrt": (3, 2),
    "power_decay": (4, 2), "mexp_decay": (5, 3), "harmonic": (6, 2),
    "exp_plus": (7, 3), "parabola": (8, 3), "const": (9, 1),
    "buckingham": (10, 3), "born": (11, 5),
    "universal": (12, 4), "eopp": (13, 6), "eopp_exp": (14, 6), "meopp": (15, 7),
    "gen_lj": (16, 5), "double_morse": (17, 7), "double_exp": (18, 5), "mishin": (19, 6),
    "poly5": (20, 5), "stiweb_2": (21, 6), "stiweb_3": (22, 2), "tersoff": (23, 11),
    "tersoff_mix": (24, 2), "tersoff_mod": (25, 16), "kawamura": (26, 9),
    "kawamura_mix": (27, 12), "softshell": (28, 2), "strmm": (29, 5),
    "lj_sc": (30, 3), "morse_sc": (31, 4), "exp_decay_sc": (32, 3), "eopp_sc": (33, 7),
}


def acsf_size(spec, nt):
    """Descriptor length of an ACSF table for nt species (AcsfLayout,
    acsf.hpp:23-33): nt(nG1 + nG2 + nG3) + npair(nG4 + nG5)."""
    g1, n2, n3, n4, n5 = (int(x) for x in spec.values[1:6])
    return nt * (g1 + n2 + n3) + nt * (nt + 1) // 2 * (n4 + n5)


def lmbtr_size(spec, nt):
    """Descriptor length of an LMBTR table for nt species (LmbtrLayout,
    lmbtr.hpp:13-38): nt·n2 + npair·n3, a term with n = 0 absent."""
    n2, n3 = int(spec.values[3]), int(spec.values[7])
    return nt * n2 + nt * (nt + 1) // 2 * n3


def descriptor_size(model):
    """Descriptor length S of an ACSF or LMBTR model."""
    spec = model.tables[0]
    return lmbtr_size(spec, model.ntypes) if model.family == FS_FAMILY_LMBTR else acsf_size(spec, model.ntypes)


class FsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"status {code}: {msg}")
        self.code = code


class fs_table(C.Structure):
    _fields_ = [("kind", C.c_int32), ("form", C.c_int32), ("n", C.c_int32),
                ("reserved", C.c_int32), ("rmin", C.c_double), ("rmax", C.c_double),
                ("values", C.POINTER(C.c_double)), ("fixed", C.POINTER(C.c_uint8)),
                ("lower", C.POINTER(C.c_double)), ("upper", C.POINTER(C.c_double))]


class fs_model(C.Structure):
    _fields_ = [("family", C.c_int32), ("ntypes", C.c_int32), ("n_tables", C.c_int32),
                ("reserved", C.c_int32), ("tables", C.POINTER(fs_table)),
                ("n_globals", C.c_int32), ("n_links", C.c_int32),
                ("global_values", C.POINTER(C.c_double)), ("global_fixed", C.POINTER(C.c_uint8)),
                ("link_global", C.POINTER(C.c_int32)), ("link_table", C.POINTER(C.c_int32)),
                ("link_param", C.POINTER(C.c_int32))]


class fs_gpu_opts(C.Structure):
    _fields_ = [("device", C.c_int32), ("precision", C.c_int32),
                ("lanes_per_atom", C.c_int32), ("reserved", C.c_int32)]


class fs_tune_report(C.Structure):
    _fields_ = [("lanes_per_atom", C.c_int32), ("k2_warps", C.c_int32), ("pop_waves", C.c_int32),
                ("reserved", C.c_int32), ("residual_ms", C.c_double * 4), ("jacobian_ms", C.c_double * 5),
                ("population_ms", C.c_double * 3)]


class fs_surrogate_opts(C.Structure):
    _fields_ = [("screen", C.c_int32), ("warm_generations", C.c_int32), ("batch", C.c_int32),
                ("steps_per_generation", C.c_int32), ("lr", C.c_double), ("gate", C.c_double),
                ("holdout", C.c_double), ("seed", C.c_uint64), ("archive_rows", C.c_int64)]


class fs_de_opts(C.Structure):
    _fields_ = [("NP", C.c_int32), ("reserved", C.c_int32), ("mutation", C.c_double),
                ("crossover", C.c_double), ("seed", C.c_uint64), ("w_e", C.c_double),
                ("w_s", C.c_double)]


def _dp(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int32))


@dataclass
class Table:
    """One table of a calculator, in the reference's gather order."""
    kind: int
    values: np.ndarray
    rmin: float = 0.0
    rmax: float = 0.0
    form: int = 0
    fixed: Optional[np.ndarray] = None
    lower: Optional[np.ndarray] = None
    upper: Optional[np.ndarray] = None

    @staticmethod
    def spline(rmin, rmax, knots, fixed=None):
        return Table(FS_TABLE_SPLINE, np.ascontiguousarray(knots, dtype=np.float64),
                     float(rmin), float(rmax), 0,
                     None if fixed is None else np.ascontiguousarray(fixed, dtype=np.uint8))

    @staticmethod
    def analytic(name, params, rmin, rmax, fixed=None, lower=None, upper=None):
        form, npar = FORMS[name]
        p = np.ascontiguousarray(params, dtype=np.float64)
        assert p.size == npar, (name, p.size, npar)
        f = lambda a, dt: None if a is None else np.ascontiguousarray(a, dtype=dt)
        return Table(FS_TABLE_ANALYTIC, p, float(rmin), float(rmax), form,
                     f(fixed, np.uint8), f(lower, np.float64), f(upper, np.float64))

    @staticmethod
    def sw(A, B, p, q, delta, a1, gamma, a2, fixed=None):
        v = np.array([A, B, p, q, delta, a1, gamma, a2], dtype=np.float64)
        return Table(FS_TABLE_SW, v, 0.0, 0.0, 0,
                     None if fixed is None else np.ascontiguousarray(fixed, dtype=np.uint8))

    @staticmethod
    def tersoff(A, B, lam, mu, beta, n, c, d, h, R, S, omega=1.0, fixed=None):
        """TersoffParams of one pair slot, in the reference's field order
        (tersoff_force.hpp:17-31); omega is fixed unless `fixed` says
        otherwise, as the reference declares it."""
        v = np.array([A, B, lam, mu, beta, n, c, d, h, R, S, omega], dtype=np.float64)
        fx = np.zeros(12, np.uint8) if fixed is None else np.ascontiguousarray(fixed, dtype=np.uint8)
        if fixed is None:
            fx[11] = 1
        return Table(FS_TABLE_TERSOFF, v, 0.0, 0.0, 0, fx)

    @staticmethod
    def acsf(rcut, g1=0, g2=(), g3=(), g4=(), g5=()):
        """ACSF symmetry functions (the reference's ACSF fields, acsf.hpp:48-71):
        g1 parameterless channels, g2 (eta, rs), g3 kappa, g4 and g5
        (eta, zeta, lambda).  Descriptor hyperparameters are not fitted."""
        v = [rcut, g1, len(g2), len(g3), len(g4), len(g5)]
        for seq in (g2, g3, g4, g5):
            for x in seq:
                v += list(np.atleast_1d(np.asarray(x, np.float64)))
        v = np.array(v, np.float64)
        return Table(FS_TABLE_ACSF, v, 0.0, 0.0, 0, np.ones(v.size, np.uint8))

    @staticmethod
    def lmbtr(rcut=6.0, weight_scale=3.0, normalize=True, k2=(0.0, 6.0, 50, 0.3), k3=(-1.0, 1.0, 50, 0.1)):
        """LMBTR descriptor (the reference's LMBTR fields and defaults,
        lmbtr.hpp:40-47): k2 and k3 grids as (min, max, n, sigma) or None
        for an absent term; distances r_ij on the k2 grid, cos θ_ijk on the
        k3 grid.  Descriptor hyperparameters are not fitted."""
        def grid(g):
            if g is None:
                return [0, 0.0, 0.0, 0.0]
            lo, hi, n, sig = g
            return [int(n), float(lo), float(hi), float(sig)]
        v = np.array([rcut, weight_scale, 1.0 if normalize else 0.0] + grid(k2) + grid(k3), np.float64)
        return Table(FS_TABLE_LMBTR, v, 0.0, 0.0, 0, np.ones(v.size, np.uint8))

    @staticmethod
    def linear_head(coeffs, bias=0.0, bias_fixed=True, fixed=None):
        """LinearHead E_i = w·D_i + b (ml_force.hpp); the bias is fixed unless
        bias_fixed is False, as the reference declares it."""
        v = np.append(np.asarray(coeffs, np.float64), float(bias))
        fx = np.zeros(v.size, np.uint8) if fixed is None else np.ascontiguousarray(fixed, np.uint8)
        if fixed is None:
            fx[-1] = 1 if bias_fixed else 0
        return Table(FS_TABLE_LINEAR_HEAD, v, 0.0, 0.0, 0, fx)

    @staticmethod
    def standardization(mean, inv_std):
        """Per-species descriptor standardization {mean[S], inv_std[S]}: the
        head sees (D − mean) ⊙ inv_std (MLBase, ml_force.hpp:607-623).  Not
        fitted: every value is fixed."""
        v = np.concatenate([np.asarray(mean, np.float64), np.asarray(inv_std, np.float64)])
        return Table(FS_TABLE_STANDARDIZATION, v, 0.0, 0.0, 0, np.ones(v.size, np.uint8))

    @staticmethod
    def lam(values, fixed=None):
        return Table(FS_TABLE_LAMBDA, np.ascontiguousarray(values, dtype=np.float64),
                     fixed=None if fixed is None else np.ascontiguousarray(fixed, dtype=np.uint8))

    def copy(self):
        c = lambda a: None if a is None else a.copy()
        return Table(self.kind, self.values.copy(), self.rmin, self.rmax, self.form,
                     c(self.fixed), c(self.lower), c(self.upper))


@dataclass
class GlobalParam:
    """A parameter shared by several analytic parameters (GlobalParam,
    include/forcesmith/force/force_calculator_concept.hpp:21-44): its value,
    fixed flag and links (table index in model order, parameter slot).  A
    linked parameter is fixed in its table and takes the global's value
    (finalize_globals, :230-237); a free global takes the column after every
    table column, in global order."""
    value: float
    fixed: bool = False
    links: list = field(default_factory=list)
    name: str = ""

    def copy(self):
        return GlobalParam(float(self.value), bool(self.fixed), [tuple(lk) for lk in self.links], self.name)


@dataclass
class Model:
    family: int
    ntypes: int
    tables: list = field(default_factory=list)
    globals: list = field(default_factory=list)

    def _free_mask(self, k):
        """Free values of table k: not fixed and not linked to a global."""
        t = self.tables[k]
        free = (t.fixed == 0) if t.fixed is not None else np.ones(t.values.size, bool)
        for g in self.globals:
            for tk, slot in g.links:
                if tk == k:
                    free[slot] = False
        return free

    def broadcast_globals(self):
        """Each linked parameter takes its global's value (in place)."""
        for g in self.globals:
            for tk, slot in g.links:
                self.tables[tk].values[slot] = g.value
        return self

    def to_c(self):
        """Returns (fs_model, keepalive) — keep the second alive while in use."""
        arr = (fs_table * len(self.tables))()
        keep = [arr]
        for k, t in enumerate(self.tables):
            ft = arr[k]
            ft.kind, ft.form, ft.n = t.kind, t.form, int(t.values.size)
            ft.rmin, ft.rmax = t.rmin, t.rmax
            ft.values = _dp(t.values)
            ft.fixed = None if t.fixed is None else t.fixed.ctypes.data_as(C.POINTER(C.c_uint8))
            ft.lower = _dp(t.lower)
            ft.upper = _dp(t.upper)
            keep.append(t)
        m = fs_model(self.family, self.ntypes, len(self.tables), 0, arr)
        if self.globals:
            gv = np.array([g.value for g in self.globals], np.float64)
            gf = np.array([1 if g.fixed else 0 for g in self.globals], np.uint8)
            links = [(gi, tk, slot) for gi, g in enumerate(self.globals) for tk, slot in g.links]
            lg, lt, lp = (np.array([lk[q] for lk in links], np.int32) for q in range(3))
            keep += [gv, gf, lg, lt, lp]
            ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
            m.n_globals, m.n_links = len(self.globals), len(links)
            m.global_values, m.global_fixed = _dp(gv), gf.ctypes.data_as(C.POINTER(C.c_uint8))
            m.link_global, m.link_table, m.link_param = ip(lg), ip(lt), ip(lp)
        return m, keep

    def with_standardization(self, mean, inv_std):
        """An ACSF or LMBTR model with the per-species standardization tables
        set to mean, inv_std (nt × S), replacing any it had."""
        assert self.family in (FS_FAMILY_ACSF, FS_FAMILY_LMBTR)
        mean, inv_std = np.asarray(mean, np.float64), np.asarray(inv_std, np.float64)
        tabs = [t.copy() for t in self.tables[:1 + self.ntypes]]
        tabs += [Table.standardization(mean[t], inv_std[t]) for t in range(self.ntypes)]
        return Model(self.family, self.ntypes, tabs)

    def acsf_remapped(self, old_species, new_species):
        """An ACSF model for the species list new_species, from this model's
        heads for old_species (MLBase::remap, ml_force.hpp:165-190):
        descriptor index k of the new layout takes the head coefficient of the
        old index that describes the same species channel (remap_layout,
        descriptor_layout.cpp:9-50); channels without an old counterpart get
        coefficient 0 with the head's first coefficient's fixed flag
        (LinearHead::remapped, ml_force.cpp:52-65).  A new species without an
        old one gets a zero head, coefficients free and bias 0 fixed
        (zero_like, :67-71).  Standardization is dropped, as remap drops it.

        As in remap_layout, a block counts as per-species when its channel
        count equals the new species count; with one new species that is also
        true of the pair blocks (one pair channel)."""
        assert self.family == FS_FAMILY_ACSF
        old_of_new = [list(old_species).index(x) if x in old_species else None for x in new_species]
        spec = self.tables[0]
        S_old, S_new = self.ntypes, len(new_species)
        g1, n2, n3, n4, n5 = (int(x) for x in spec.values[1:6])

        def layout(nt):  # (base, count, nchan) per block: G1..G3 per species, G4, G5 per pair
            P, base, out = nt * (nt + 1) // 2, 0, []
            for count, nch in ((g1, nt), (n2, nt), (n3, nt), (n4, P), (n5, P)):
                out.append((base, count, nch))
                base += count * nch
            return out, base

        def ordinal(a, b, nt):  # pair_ordinal: upper triangle, row-major
            a, b = min(a, b), max(a, b)
            return a * nt - a * (a - 1) // 2 + (b - a)

        Lo, _ = layout(S_old)
        Ln, size = layout(S_new)
        idx = [None] * size
        for (bo, _, _), (bn, count, nch) in zip(Lo, Ln):
            if nch == S_new:  # per species
                for sn, so in enumerate(old_of_new):
                    if so is not None:
                        for t in range(count):
                            idx[bn + sn * count + t] = bo + so * count + t
            else:  # per pair
                for a in range(S_new):
                    for c in range(a, S_new):
                        ao, co = old_of_new[a], old_of_new[c]
                        if ao is None or co is None:
                            continue
                        pn, po = ordinal(a, c, S_new), ordinal(ao, co, S_old)
                        for t in range(count):
                            idx[bn + pn * count + t] = bo + po * count + t
        heads = []
        for so in old_of_new:
            if so is None:
                fx = np.zeros(size + 1, np.uint8)
                fx[-1] = 1
                heads.append(Table.linear_head(np.zeros(size), 0.0, fixed=fx))
                continue
            h = self.tables[1 + so]
            hv = h.values
            hf = h.fixed if h.fixed is not None else np.zeros(hv.size, np.uint8)
            f0 = hf[0] if hv.size > 1 else 0
            v = np.zeros(size + 1)
            fx = np.full(size + 1, f0, np.uint8)
            for k, src in enumerate(idx):
                if src is not None:
                    v[k], fx[k] = hv[src], hf[src]
            v[-1], fx[-1] = hv[-1], hf[-1]
            heads.append(Table.linear_head(v[:-1], v[-1], fixed=fx))
        return Model(FS_FAMILY_ACSF, S_new, [spec.copy()] + heads)

    def free_values(self) -> np.ndarray:
        """The parameter vector in gather order: every table's free values,
        then the free globals (force_calculator_concept.hpp:171-208)."""
        out = [t.values[self._free_mask(k)] for k, t in enumerate(self.tables)]
        out.append(np.array([g.value for g in self.globals if not g.fixed], np.float64))
        return np.concatenate(out)

    def with_values(self, x: np.ndarray) -> "Model":
        """scatter_params: a copy with x placed in gather order and the
        globals broadcast to their links."""
        m = self.copy()
        o = 0
        for k, t in enumerate(m.tables):
            free = m._free_mask(k)
            n = int(free.sum())
            t.values[free] = x[o:o + n]
            o += n
        for g in m.globals:
            if not g.fixed:
                g.value = float(x[o])
                o += 1
        return m.broadcast_globals()

    def copy(self):
        return Model(self.family, self.ntypes, [t.copy() for t in self.tables], [g.copy() for g in self.globals])


@dataclass
class Dataset:
    """Concatenated periodic configurations (shapes of fs_gpu_upload_configs)."""
    natoms: np.ndarray            # int32[n_cfg]
    box9: np.ndarray              # float64[n_cfg, 9] row-major, lattice vectors as columns
    pos: np.ndarray               # float64[N, 3]
    type: np.ndarray              # int32[N]
    ref_force: Optional[np.ndarray] = None   # float64[N, 3]
    ref_energy: Optional[np.ndarray] = None  # float64[n_cfg]
    ref_stress9: Optional[np.ndarray] = None  # float64[n_cfg, 9]

    @property
    def n_cfg(self):
        return int(self.natoms.size)

    @property
    def n_atoms(self):
        return int(self.natoms.sum())

    def rows(self, w_s: float) -> int:
        return int(3 * self.n_atoms + self.n_cfg * (2 + (6 if w_s > 0 else 0)))

    def subset(self, idx):
        idx = np.asarray(idx)
        starts = np.concatenate([[0], np.cumsum(self.natoms)])
        sel = np.concatenate([np.arange(starts[i], starts[i + 1]) for i in idx]) \
            if idx.size else np.zeros(0, np.int64)
        g = lambda a, s: None if a is None else np.ascontiguousarray(a[s])
        return Dataset(np.ascontiguousarray(self.natoms[idx]), np.ascontiguousarray(self.box9[idx]),
                       np.ascontiguousarray(self.pos[sel]), np.ascontiguousarray(self.type[sel]),
                       g(self.ref_force, sel), g(self.ref_energy, idx), g(self.ref_stress9, idx))

    def with_types(self, type_):
        return Dataset(self.natoms, self.box9, self.pos, np.ascontiguousarray(type_, np.int32),
                       self.ref_force, self.ref_energy, self.ref_stress9)

    def with_labels(self, forces, energy, stress9):
        return Dataset(self.natoms, self.box9, self.pos, self.type,
                       np.ascontiguousarray(forces, np.float64).reshape(-1, 3),
                       np.ascontiguousarray(energy, np.float64),
                       np.ascontiguousarray(stress9, np.float64).reshape(-1, 9))


class Session:
    """Handle-based wrapper over an `fs_gpu_*`-shaped C ABI (`prefix_*`)."""

    def __init__(self, lib: C.CDLL, prefix: str, handle: C.c_void_p, err_fn=None):
        self._lib = lib
        self._p = prefix
        self._h = handle
        self._err_fn = err_fn
        self._keep = None
        self.D = None

    def _f(self, name):
        return getattr(self._lib, f"{self._p}_{name}")

    def _check(self, rc, what):
        if rc != FS_OK:
            msg = what
            if self._err_fn is not None:
                msg = f"{what}: {self._err_fn(self._h)}"
            raise FsError(rc, msg)

    def upload(self, ds: Dataset):
        self._ds = ds
        rc = self._f("upload_configs")(self._h, C.c_int32(ds.n_cfg), _ip(ds.natoms),
                                       _dp(np.ascontiguousarray(ds.box9, np.float64)),
                                       _dp(np.ascontiguousarray(ds.pos, np.float64)), _ip(ds.type),
                                       _dp(ds.ref_force), _dp(ds.ref_energy), _dp(ds.ref_stress9))
        self._check(rc, "upload_configs")

    def set_references(self, ds: Dataset):
        rc = self._f("set_references")(self._h, _dp(ds.ref_force), _dp(ds.ref_energy),
                                       _dp(ds.ref_stress9))
        self._check(rc, "set_references")

    def set_model(self, model: Model, prepare=True):
        m, keep = model.to_c()
        self._keep = keep
        self._model = model
        self._check(self._f("set_model")(self._h, C.byref(m)), "set_model")
        d = C.c_int32()
        self._check(self._f("param_count")(self._h, C.byref(d)), "param_count")
        self.D = d.value
        if prepare:
            self._check(self._f("prepare")(self._h), "prepare")

    def prepare(self):
        self._check(self._f("prepare")(self._h), "prepare")

    def acsf_standardization(self):
        """ACSF and LMBTR models: per-species descriptor mean and 1/σ over
        every uploaded atom, and the atoms per species
        (MLBase::compute_standardization).  Returns (mean nt × S, inv_std
        nt × S, count nt)."""
        nt = self._model.ntypes
        S = descriptor_size(self._model)
        mean, inv_std = np.zeros((nt, S)), np.zeros((nt, S))
        count = np.zeros(nt, np.int64)
        self._check(self._f("acsf_standardization")(self._h, _dp(mean), _dp(inv_std),
                                                    count.ctypes.data_as(C.POINTER(C.c_int64))),
                    "acsf_standardization")
        return mean, inv_std, count

    def num_pairs(self):
        n = C.c_int64()
        self._check(self._f("num_pairs")(self._h, C.byref(n)), "num_pairs")
        return n.value

    def neighbor_counts(self, n_atoms):
        out = np.zeros(n_atoms, np.int32)
        self._check(self._f("get_neighbor_counts")(self._h, _ip(out)), "get_neighbor_counts")
        return out

    def gather_params(self):
        x = np.zeros(self.D, np.float64)
        self._check(self._f("gather_params")(self._h, _dp(x)), "gather_params")
        return x

    def gather_bounds(self):
        lo = np.zeros(self.D, np.float64)
        hi = np.zeros(self.D, np.float64)
        self._check(self._f("gather_bounds")(self._h, _dp(lo), _dp(hi)), "gather_bounds")
        return lo, hi

    def set_params(self, x):
        x = np.ascontiguousarray(x, np.float64)
        self._check(self._f("set_params")(self._h, _dp(x), C.c_int32(x.size)), "set_params")

    def residual_count(self, w_s):
        m = C.c_int64()
        self._check(self._f("residual_count")(self._h, C.c_double(w_s), C.byref(m)),
                    "residual_count")
        return m.value

    def eval(self, w_e=1.0, w_s=0.0, want=("F", "forces", "energy", "stress", "limit", "obj")):
        ds = self._ds
        m = self.residual_count(w_s)
        out = {}
        F = np.zeros(m) if "F" in want else None
        fo = np.zeros((ds.n_atoms, 3)) if "forces" in want else None
        en = np.zeros(ds.n_cfg) if "energy" in want else None
        st = np.zeros((ds.n_cfg, 9)) if "stress" in want else None
        li = np.zeros(ds.n_cfg) if "limit" in want else None
        ob = C.c_double()
        rc = self._f("eval")(self._h, C.c_double(w_e), C.c_double(w_s), _dp(F), _dp(fo), _dp(en),
                             _dp(st), _dp(li), C.byref(ob) if "obj" in want else None)
        self._check(rc, "eval")
        for k, v in (("F", F), ("forces", fo), ("energy", en), ("stress", st), ("limit", li)):
            if v is not None:
                out[k] = v
        if "obj" in want:
            out["obj"] = ob.value
        return out


def load_library(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    return C.CDLL(path, mode=C.RTLD_GLOBAL)
