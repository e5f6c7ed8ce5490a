"""Forcesmith's data formats on either side of the device path.

  read_configs / write_configs  the configuration JSON of
      src/io/config_reader.cpp:58-200 — a top-level array of
      {name?, X, Y, Z, E, W?, S?, atoms: [{element, position, force?}]};
      the box's lattice vectors are X, Y, Z (its columns), S is the stress
      in the order xx, yy, zz, xy, yz, xz (config_reader.cpp:78-91), and the
      species slots are the elements present sorted by atomic number (the
      species registry, species.hpp).
  read_model / write_model  the force-model JSON of
      src/io/force_model_reader.cpp:134-440 for the families this path
      evaluates: a bare pair file (no "model" key; the pair count fixes
      ntypes), and "pair", "eam", "adp" (table sections "pair", "density",
      "embedding", "dipole", "quadrupole"), "stiweb" ("potentials": SWParams
      objects, "lambda").  A table section is {"format", "potentials": [...]}
      with tabulated {rmin, rmax, knots, fixed?} or analytic {type, rmin,
      rmax, <parameter>: number | {value, min?, max?, fixed?}} entries
      (src/io/potential_reader.cpp:60-200).  Pair and EAM models may carry
      global parameters: {"globals": {name: {value, fixed?}}} and
      {"global": name} in place of an analytic parameter
      (force_model_reader.cpp:59-117).
  read_potential  a bare potential section → list of tables
      (parse_potential, src/io/potential_reader.cpp).
  write_native / write_lammps / write_imd / write_model_file  the sampled
      writers of src/io/output_writer.cpp and write_model.cpp: every radial
      table on 500 uniform points of its span, values (and derivatives for
      LAMMPS) from a sampler — fs_gpu_tabulate on the device through
      session_sampler.
  read_setfl  a single-element LAMMPS setfl file as three makima tables on
      the file's own grids (φ = r·φ / r from the second r point on).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from .abi import (FS_FAMILY_ACSF, FS_FAMILY_LMBTR, FS_FAMILY_ADP, FS_FAMILY_ANGULAR, FS_FAMILY_EAM, FS_FAMILY_PAIR,
                  FS_FAMILY_SW, FS_FAMILY_TERSOFF, FS_TABLE_ANALYTIC, FS_TABLE_LAMBDA, FS_TABLE_SPLINE,
                  FS_TABLE_SW, FS_TABLE_TERSOFF, FORMS, TERSOFF_FIELDS, Dataset, GlobalParam, Model, Table,
                  acsf_size, descriptor_size, lmbtr_size)

SYMBOLS = (
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
    "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm "
    "Yb Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No "
    "Lr Rf Db Sg Bh Hs Mt Ds Rg Cn Nh Fl Mc Lv Ts Og").split()
Z_OF = {s: z + 1 for z, s in enumerate(SYMBOLS)}

# analytic form names (and aliases) and parameter names, as the reference spells them
_TERSOFF_P = ("A", "B", "lambda", "mu", "beta", "n", "c", "d", "h", "R", "S")
_EOPP_P = ("A", "n", "B", "m", "k", "phi")
_KAW_P = ("A", "B", "C", "D", "E", "F", "G", "H", "I")
# canonical name: (aliases, parameter names), analytic_potential.hpp:304-806
_FORMS = {
    "lj": (("pair_lj",), ("epsilon", "sigma")),
    "morse": ((), ("De", "a", "re")),
    "exp_decay": (("exp",), ("A", "B")),
    "sqrt": ((), ("A", "B")),
    "power_decay": (("power",), ("A", "n")),
    "mexp_decay": (("mexp",), ("A", "B", "r0")),
    "harmonic": ((), ("k", "r0")),
    "exp_plus": (("expplus",), ("A", "B", "C")),
    "parabola": ((), ("A", "B", "C")),
    "const": ((), ("C",)),
    "buckingham": (("buck",), ("A", "rho", "C")),
    "born": ((), ("A", "B", "C", "D", "E")),
    "universal": ((), ("E0", "a", "b", "c")),
    "eopp": ((), _EOPP_P),
    "eopp_exp": (("eopp_exp_",), ("A", "B", "C", "m", "k", "phi")),
    "meopp": ((), ("A", "n", "B", "m", "k", "phi", "r0")),
    "gen_lj": (("genlj",), ("A", "n", "m", "r0", "B")),
    "double_morse": (("dbl_morse",), ("D1", "a1", "r1", "D2", "a2", "r2", "C")),
    "double_exp": (("dbl_exp",), ("A", "B", "r1", "C", "r2")),
    "mishin": ((), ("A", "B", "C", "r0", "n", "d")),
    "poly5": ((), ("a0", "a1", "a2", "a3", "a4")),
    "stiweb_2": (("sw2",), ("A", "B", "p", "q", "delta", "rc")),
    "stiweb_3": (("sw3",), ("gamma", "a")),
    "tersoff": (("tersoff_pot",), _TERSOFF_P),
    "tersoff_mix": ((), ("chi", "omega")),
    "tersoff_mod": (("tmod",), _TERSOFF_P + ("c1", "c2", "c3", "c4", "c5")),
    "kawamura": ((), _KAW_P),
    "kawamura_mix": ((), _KAW_P + ("J", "K", "L")),
    "softshell": (("soft",), ("A", "n")),
    "strmm": ((), ("A", "B", "C", "D", "E")),
    "lj_sc": (("pair_lj_sc",), ("epsilon", "sigma", "h")),
    "morse_sc": ((), ("De", "a", "re", "h")),
    "exp_decay_sc": (("exp_sc",), ("A", "B", "h")),
    "eopp_sc": ((), _EOPP_P + ("h",)),
}
# every spelling the reference accepts: name or alias → (canonical name, parameter names)
FORM_SPEC = {alias: (canon, names) for canon, (aliases, names) in _FORMS.items()
             for alias in (canon,) + aliases}
FORM_NAME = {FORMS[canon][0]: canon for canon, _ in FORM_SPEC.values()}
PARAM_NAMES = {FORMS[canon][0]: names for canon, names in FORM_SPEC.values()}
SW_FIELDS = ("A", "B", "p", "q", "delta", "a1", "gamma", "a2")
# table sections per family (family_name, include/forcesmith/core/families.hpp:28-43;
# the TableField lists of the calculators, e.g. angular_force.hpp:21-30)
TABLE_KEYS = {FS_FAMILY_PAIR: ("pair",), FS_FAMILY_EAM: ("pair", "density", "embedding"),
              FS_FAMILY_ADP: ("pair", "density", "embedding", "dipole", "quadrupole"),
              FS_FAMILY_ANGULAR: ("pair", "radial", "angular")}
PER_PAIR = {"pair": True, "density": False, "embedding": False, "dipole": True, "quadrupole": True,
            "radial": True, "angular": False}
FAMILY_OF = {"pair": FS_FAMILY_PAIR, "eam": FS_FAMILY_EAM, "adp": FS_FAMILY_ADP, "stiweb": FS_FAMILY_SW,
             "angular": FS_FAMILY_ANGULAR, "tersoff": FS_FAMILY_TERSOFF}
NAME_OF = {v: k for k, v in FAMILY_OF.items()}


class FormatError(ValueError):
    pass


def _text(src):
    if isinstance(src, (str, os.PathLike)) and os.path.exists(src):
        with open(src) as f:
            return f.read()
    return src


def _json(src):
    """Parsed JSON, with a syntax error reported as a FormatError."""
    try:
        return json.loads(_text(src))
    except json.JSONDecodeError as e:
        raise FormatError(f"invalid JSON: {e}") from None


def _vec3(v, what):
    try:
        a = np.asarray(v, np.float64)
    except (TypeError, ValueError):
        raise FormatError(f"{what}: must be an array of 3 numbers") from None
    if a.shape != (3,):
        raise FormatError(f"{what}: must be an array of 3 numbers")
    return a


# ---------------------------------------------------------------------------
# configurations

def species_slots(symbols):
    """The species registry: the distinct elements sorted by atomic number."""
    unknown = [s for s in symbols if s not in Z_OF]
    if unknown:
        raise FormatError(f"unknown element symbol(s): {unknown}")
    return sorted(set(symbols), key=lambda s: Z_OF[s])


def read_configs(src):
    """Configuration JSON → (Dataset, species symbols by slot, names, weights)."""
    j = _json(src)
    if not isinstance(j, list):
        raise FormatError("top-level JSON must be an array of configurations")
    syms = [a["element"] for c in j if isinstance(c, dict) for a in c.get("atoms", [])
            if isinstance(a, dict) and isinstance(a.get("element"), str)]
    slots = species_slots(syms)
    slot_of = {s: k for k, s in enumerate(slots)}
    natoms, box9, pos, typ, frc, ene, st9, names, weights = [], [], [], [], [], [], [], [], []
    for ci, c in enumerate(j):
        ctx = f"config[{ci}]"
        if not isinstance(c, dict):
            raise FormatError(f"{ctx}: each configuration must be a JSON object")
        for k in ("X", "Y", "Z", "E", "atoms"):
            if k not in c:
                raise FormatError(f"{ctx}: missing key '{k}'")
        cols = [_vec3(c[k], f"{ctx} '{k}'") for k in ("X", "Y", "Z")]
        box9.append(np.stack(cols, axis=1).ravel())  # lattice vectors as columns, row-major
        ene.append(float(c["E"]))
        weights.append(float(c.get("W", 1.0)))
        names.append(c.get("name", ""))
        s = np.zeros((3, 3))
        if "S" in c:
            v = np.asarray(c["S"], np.float64)
            if v.shape != (6,):
                raise FormatError(f"{ctx} 'S': must be an array of 6 doubles")
            s[0, 0], s[1, 1], s[2, 2] = v[0], v[1], v[2]
            s[0, 1] = s[1, 0] = v[3]
            s[1, 2] = s[2, 1] = v[4]
            s[0, 2] = s[2, 0] = v[5]
        st9.append(s.ravel())
        atoms = c["atoms"]
        if not isinstance(atoms, list):
            raise FormatError(f"{ctx}: 'atoms' must be an array")
        natoms.append(len(atoms))
        for ai, a in enumerate(atoms):
            if "element" not in a or "position" not in a:
                raise FormatError(f"{ctx} atom[{ai}]: needs 'element' and 'position'")
            typ.append(slot_of[a["element"]])
            pos.append(_vec3(a["position"], f"{ctx} atom[{ai}] 'position'"))
            frc.append(_vec3(a.get("force", (0.0, 0.0, 0.0)), f"{ctx} atom[{ai}] 'force'"))
    ds = Dataset(np.asarray(natoms, np.int32), np.asarray(box9).reshape(-1, 9),
                 np.asarray(pos).reshape(-1, 3), np.asarray(typ, np.int32), np.asarray(frc).reshape(-1, 3),
                 np.asarray(ene), np.asarray(st9).reshape(-1, 9))
    return ds, slots, names, np.asarray(weights)


def write_configs(ds, slots, names=None, weights=None):
    """Dataset → configuration JSON text (the inverse of read_configs)."""
    out, a0 = [], 0
    for c in range(ds.n_cfg):
        b = np.asarray(ds.box9[c]).reshape(3, 3)
        s = np.asarray(ds.ref_stress9[c]).reshape(3, 3)
        n = int(ds.natoms[c])
        atoms = [{"element": slots[int(ds.type[a0 + k])], "position": [float(v) for v in ds.pos[a0 + k]],
                  "force": [float(v) for v in ds.ref_force[a0 + k]]} for k in range(n)]
        cfg = {"X": b[:, 0].tolist(), "Y": b[:, 1].tolist(), "Z": b[:, 2].tolist(),
               "E": float(ds.ref_energy[c]),
               "S": [s[0, 0], s[1, 1], s[2, 2], s[0, 1], s[1, 2], s[0, 2]], "atoms": atoms}
        if names is not None:
            cfg["name"] = names[c]
        if weights is not None:
            cfg["W"] = float(weights[c])
        out.append(cfg)
        a0 += n
    return json.dumps(out, indent=1)


# ---------------------------------------------------------------------------
# models

def _param(v):
    if isinstance(v, dict):
        if "value" not in v:
            raise FormatError("parameter object missing 'value'")
        lo, hi = float(v.get("min", -math.inf)), float(v.get("max", math.inf))
        if lo > hi:
            raise FormatError("parameter has min > max")
        return float(v["value"]), lo, hi, bool(v.get("fixed", False))
    return float(v), -math.inf, math.inf, False


def _potential(p):
    if not isinstance(p, dict):
        raise FormatError("potential spec must be a JSON object")
    if "type" in p:
        if p["type"] not in FORM_SPEC:
            raise FormatError(f"unknown analytic function: {p['type']}")
        canon, names = FORM_SPEC[p["type"]]
        vals = []
        for nm in names:
            if nm not in p:
                raise FormatError(f"missing parameter '{nm}' for type {p['type']}")
            vals.append(_param(p[nm]))
        v = np.array([x[0] for x in vals])
        return Table.analytic(canon, v, float(p["rmin"]), float(p["rmax"]),
                              fixed=np.array([x[3] for x in vals], np.uint8),
                              lower=np.array([x[1] for x in vals]), upper=np.array([x[2] for x in vals]))
    if "knots" in p:
        knots = p["knots"]
        if not isinstance(knots, list) or not all(
                isinstance(v, (int, float)) and not isinstance(v, bool) for v in knots):
            raise FormatError("tabulated potential: 'knots' must be an array of numbers")
        y = np.asarray(knots, np.float64)
        if y.size < 2:
            raise FormatError("tabulated potential needs at least 2 knots")
        rmin, rmax = float(p["rmin"]), float(p["rmax"])
        if not rmax > rmin:
            raise FormatError(f"tabulated potential requires rmax > rmin (got rmin={rmin}, rmax={rmax})")
        fixed = np.ones(y.size, np.uint8) if p.get("fixed", False) else None
        return Table.spline(rmin, rmax, y, fixed=fixed)
    raise FormatError("potential spec has neither 'type' (analytic) nor 'knots' (tabulated)")


def _section(sub, want, label):
    if "format" not in sub:
        raise FormatError(f"{label}: missing 'format' key")
    if sub["format"] not in ("analytic", "tabulated"):
        raise FormatError(f"{label}: unsupported potential format '{sub['format']}'")
    pots = sub.get("potentials")
    if not isinstance(pots, list):
        raise FormatError(f"{label}: missing or invalid 'potentials' array")
    if len(pots) != want:
        raise FormatError(f"{label}: expected {want} potentials, got {len(pots)}")
    return [_potential(p) for p in pots]


def read_potential(src):
    """A potential section {"format", "potentials": [...]} → list of Tables
    (parse_potential, src/io/potential_reader.cpp)."""
    j = _json(src)
    if not isinstance(j, dict):
        raise FormatError("potential file must be a JSON object")
    pots = j.get("potentials")
    return _section(j, len(pots) if isinstance(pots, list) else -1, "potential")


def _build_globals(j, regions):
    """build_globals (src/io/force_model_reader.cpp:59-117): the "globals"
    object {name: {value, fixed?}} (min and max are not read), then every
    analytic parameter given as {"global": name} in the region sections is
    linked to that global and replaced by its seed value.  regions: (section
    JSON, first table index of the section)."""
    out, by_name = [], {}
    for gname, spec in (j.get("globals") or {}).items():
        if not isinstance(spec, dict) or "value" not in spec:
            raise FormatError(f"globals: global '{gname}' missing 'value'")
        by_name[gname] = len(out)
        out.append(GlobalParam(float(spec["value"]), bool(spec.get("fixed", False)), [], gname))
    for sub, t0 in regions:
        pots = sub.get("potentials") if isinstance(sub, dict) else None
        if not isinstance(pots, list):
            continue
        for i, pot in enumerate(pots):
            if not isinstance(pot, dict) or "type" not in pot:
                continue
            for key in [k for k, v in pot.items() if isinstance(v, dict) and "global" in v]:
                gname = pot[key]["global"]
                if gname not in by_name:
                    raise FormatError(f"globals: reference to undefined global '{gname}'")
                spec = FORM_SPEC.get(pot["type"])
                if spec is None or key not in spec[1]:
                    raise FormatError(f"globals: global ref on parameter '{key}' not valid for analytic "
                                      f"type '{pot['type']}'")
                g = out[by_name[gname]]
                g.links.append((t0 + i, spec[1].index(key)))
                pot[key] = g.value
    return out


def read_model(src):
    """Force-model JSON → Model (families pair, eam, adp, angular, stiweb,
    tersoff, and ml with an ACSF descriptor and linear heads).  Pair and EAM
    models may carry global parameters ("globals")."""
    j = _json(src)
    if not isinstance(j, dict):
        raise FormatError("force-model file must be a JSON object")
    if "model" not in j:
        count = len(j.get("potentials", [])) if isinstance(j.get("potentials"), list) else 0
        nt = 1
        while nt * (nt + 1) // 2 < count:
            nt += 1
        if nt * (nt + 1) // 2 != count:
            raise FormatError(f"bare pair file: {count} potentials is not a valid pair count for any ntypes")
        glob = _build_globals(j, [(j, 0)])
        return _finish_globals(Model(FS_FAMILY_PAIR, nt, _section(j, count, "pair")), glob)
    name = j["model"]
    if name == "ml":
        return _read_ml(j)
    if name not in FAMILY_OF:
        raise FormatError(f"unsupported model '{name}'")
    fam, nt = FAMILY_OF[name], int(j.get("ntypes", 1))
    npair = nt * (nt + 1) // 2
    if fam == FS_FAMILY_TERSOFF:
        # build_tersoff (src/io/force_model_reader.cpp:166-196): one parameter
        # block per pair slot; ω is free only when the block gives it
        pots = j.get("potentials")
        if not isinstance(pots, list) or len(pots) != npair:
            raise FormatError(f"tersoff: expected {npair} entries for ntypes={nt}")
        tabs = []
        for p in pots:
            if not isinstance(p, dict):
                raise FormatError("tersoff: parameter block must be a JSON object")
            vals = []
            for k in TERSOFF_FIELDS:
                if k in p:
                    vals.append(_param(p[k]))
                elif k == "omega":
                    vals.append((1.0, -math.inf, math.inf, True))
                else:
                    raise FormatError(f"tersoff: missing parameter '{k}'")
            tabs.append(Table(FS_TABLE_TERSOFF, np.array([v[0] for v in vals]), 0.0, 0.0, 0,
                              np.array([v[3] for v in vals], np.uint8), np.array([v[1] for v in vals]),
                              np.array([v[2] for v in vals])))
        return Model(fam, nt, tabs)
    if fam == FS_FAMILY_SW:
        pots = j.get("potentials")
        if not isinstance(pots, list) or len(pots) != npair:
            raise FormatError(f"stiweb: expected {npair} entries for ntypes={nt}")
        tabs = []
        for p in pots:
            vals = [_param(p[k]) for k in SW_FIELDS]
            tabs.append(Table(FS_TABLE_SW, np.array([v[0] for v in vals]), 0.0, 0.0, 0,
                              np.array([v[3] for v in vals], np.uint8), np.array([v[1] for v in vals]),
                              np.array([v[2] for v in vals])))
        lam = j.get("lambda")
        if not isinstance(lam, list) or len(lam) != nt * npair:
            raise FormatError(f"stiweb: expected {nt * npair} lambda entries for ntypes={nt}")
        vals = [_param(v) for v in lam]
        tabs.append(Table(FS_TABLE_LAMBDA, np.array([v[0] for v in vals]), 0.0, 0.0, 0,
                          np.array([v[3] for v in vals], np.uint8), np.array([v[1] for v in vals]),
                          np.array([v[2] for v in vals])))
        return Model(fam, nt, tabs)
    subs, regions, t0 = [], [], 0
    for key in TABLE_KEYS[fam]:
        sub = j if (name == "pair" and key == "pair" and "pair" not in j) else j.get(key)
        if sub is None:
            raise FormatError(f"{name}: missing section '{key}'")
        n = npair if PER_PAIR[key] else nt
        subs.append((sub, n, f"{name}.{key}"))
        regions.append((sub, t0))
        t0 += n
    # global parameters belong to the pair and EAM calculators (with_globals<>,
    # pair_force.hpp:27, eam_force.hpp:18)
    glob = _build_globals(j, regions) if fam in (FS_FAMILY_PAIR, FS_FAMILY_EAM) else []
    tabs = []
    for sub, n, label in subs:
        tabs += _section(sub, n, label)
    return _finish_globals(Model(fam, nt, tabs), glob)


def _finish_globals(model, glob):
    """finalize_globals (force_calculator_concept.hpp:230-237): linked
    parameters fixed, then every global broadcast to its links."""
    model.globals = glob
    for g in glob:
        for tk, slot in g.links:
            t = model.tables[tk]
            if t.fixed is None:
                t.fixed = np.zeros(t.values.size, np.uint8)
            t.fixed[slot] = 1
            if t.lower is not None:
                t.lower[slot] = -math.inf
            if t.upper is not None:
                t.upper[slot] = math.inf
    return model.broadcast_globals()


def _pot_json(t, refs=None):
    """One potential entry; refs maps a parameter slot to the name of the
    global it is linked to (written as {"global": name})."""
    refs = refs or {}
    if t.kind == FS_TABLE_SPLINE:
        d = {"rmin": t.rmin, "rmax": t.rmax, "knots": [float(v) for v in t.values]}
        if t.fixed is not None and np.all(t.fixed):
            d["fixed"] = True
        return d
    name = FORM_NAME[t.form]
    d = {"type": name, "rmin": t.rmin, "rmax": t.rmax}
    for k, nm in enumerate(PARAM_NAMES[t.form]):
        if k in refs:
            d[nm] = {"global": refs[k]}
            continue
        lo = -math.inf if t.lower is None else float(t.lower[k])
        hi = math.inf if t.upper is None else float(t.upper[k])
        fx = False if t.fixed is None else bool(t.fixed[k])
        if math.isinf(lo) and math.isinf(hi) and not fx:
            d[nm] = float(t.values[k])
        else:
            d[nm] = {"value": float(t.values[k]), "fixed": fx,
                     **({} if math.isinf(lo) else {"min": lo}), **({} if math.isinf(hi) else {"max": hi})}
    return d


def _read_ml(j):
    """build_ml / finish_ml / parse_linear_head (src/io/force_model_reader.cpp:
    217-389): an ACSF ("acsf" or "symmetry_functions") or LMBTR descriptor and
    one linear head per species."""
    nt = int(j.get("ntypes", 1))
    desc = j.get("descriptor")
    if not isinstance(desc, dict) or not isinstance(desc.get("type"), str):
        raise FormatError("ml: missing 'descriptor' object with a string 'type'")
    if desc["type"] == "lmbtr":
        spec = _read_lmbtr(desc)
        return _read_heads(j, FS_FAMILY_LMBTR, nt, spec, lmbtr_size(spec, nt))
    if desc["type"] not in ("acsf", "symmetry_functions"):
        raise FormatError(f"ml: unknown descriptor type '{desc['type']}' (acsf and lmbtr are built; soap is not)")
    g1 = desc.get("g1", 0)
    g1 = len(g1) if isinstance(g1, list) else int(g1) if isinstance(g1, (int, float)) else 0
    g2 = [(float(g["eta"]), float(g.get("rs", 0.0))) for g in desc.get("g2", [])]
    g3 = [float(g.get("kappa", 1.0)) for g in desc.get("g3", [])]
    g4 = [(float(g.get("eta", 1.0)), float(g.get("zeta", 1.0)), float(g.get("lambda", 1.0))) for g in desc.get("g4", [])]
    g5 = [(float(g.get("eta", 1.0)), float(g.get("zeta", 1.0)), float(g.get("lambda", 1.0))) for g in desc.get("g5", [])]
    spec = Table.acsf(float(desc.get("rcut", 6.0)), g1, g2, g3, g4, g5)
    S = acsf_size(spec, nt)
    if S == 0:
        raise FormatError("ml: acsf descriptor needs at least one of g1/g2/g3/g4/g5")
    return _read_heads(j, FS_FAMILY_ACSF, nt, spec, S)


def _read_lmbtr(desc):
    """The lmbtr branch of build_ml (force_model_reader.cpp:350-382): rcut
    (6), weight_scale (rcut/2), normalize (true); k2 and k3 grids {min, max,
    n, sigma} defaulting to (0, rcut, 50, 0.3) and (−1, 1, 50, 0.1); naming
    either grid drops the one not named."""
    rcut = float(desc.get("rcut", 6.0))
    ws = float(desc.get("weight_scale", rcut / 2.0))
    norm = bool(desc.get("normalize", True))

    def grid(key, lo, hi, n, sig):
        g = desc.get(key)
        if isinstance(g, dict):
            lo, hi = float(g.get("min", lo)), float(g.get("max", hi))
            n, sig = int(g.get("n", n)), float(g.get("sigma", sig))
        return (lo, hi, n, sig)

    named = "k2" in desc or "k3" in desc
    k2 = grid("k2", 0.0, rcut, 50, 0.3) if (not named or "k2" in desc) else None
    k3 = grid("k3", -1.0, 1.0, 50, 0.1) if (not named or "k3" in desc) else None
    if (k2[2] if k2 else 0) + (k3[2] if k3 else 0) <= 0:
        raise FormatError("ml: lmbtr descriptor needs k2 and/or k3 with n > 0")
    return Table.lmbtr(rcut, ws, norm, k2, k3)


def _read_heads(j, family, nt, spec, S):
    """finish_ml / parse_linear_head: one linear head per species, then the
    optional per-species standardization."""
    heads = j.get("heads")
    if not isinstance(heads, list) or len(heads) != nt:
        raise FormatError(f"ml: expected {nt} heads")
    tabs = [spec]
    for h in heads:
        if h.get("type", "linear") != "linear":
            raise FormatError(f"ml: unknown head type '{h.get('type')}'")
        co = h.get("coeffs")
        if not isinstance(co, list) or len(co) != S:
            raise FormatError(f"ml: head coeffs length != descriptor size {S}")
        fixed = np.zeros(S + 1, np.uint8)
        fixed[:S] = 1 if h.get("fixed", False) else 0
        fixed[S] = 1 if h.get("bias_fixed", True) else 0
        tabs.append(Table.linear_head(co, float(h.get("bias", 0.0)), fixed=fixed))
    model = Model(family, nt, tabs)
    if "standardization" in j:
        # finish_ml (force_model_reader.cpp:261-281): one {mean, inv_std} per
        # species, empty for a species without training atoms (identity here)
        st = j["standardization"]
        if not isinstance(st, list) or len(st) != nt:
            raise FormatError(f"ml: standardization must be an array of {nt} entries")
        mean, inv_std = np.zeros((nt, S)), np.ones((nt, S))
        for t, e in enumerate(st):
            mu, iv = e.get("mean", []), e.get("inv_std", [])
            if len(mu) != len(iv) or (mu and len(mu) != S):
                raise FormatError(f"ml: standardization mean/inv_std length {len(mu)} != descriptor size {S}")
            if mu:
                mean[t], inv_std[t] = mu, iv
        model = model.with_standardization(mean, inv_std)
    return model


def _write_ml(model):
    v = model.tables[0].values
    if model.family == FS_FAMILY_LMBTR:  # write_native for LMBTR (output_writer.cpp:238-267)
        desc = {"type": "lmbtr", "rcut": float(v[0]), "weight_scale": float(v[1]), "normalize": bool(v[2] != 0.0)}
        for key, o in (("k2", 3), ("k3", 7)):
            if int(v[o]) > 0:
                desc[key] = {"min": float(v[o + 1]), "max": float(v[o + 2]), "n": int(v[o]), "sigma": float(v[o + 3])}
    else:
        g1, n2, n3, n4, n5 = (int(x) for x in v[1:6])
        p = list(v[6:])
        g2 = [{"eta": p.pop(0), "rs": p.pop(0)} for _ in range(n2)]
        g3 = [{"kappa": p.pop(0)} for _ in range(n3)]
        g4 = [{"eta": p.pop(0), "zeta": p.pop(0), "lambda": p.pop(0)} for _ in range(n4)]
        g5 = [{"eta": p.pop(0), "zeta": p.pop(0), "lambda": p.pop(0)} for _ in range(n5)]
        desc = {"type": "acsf", "rcut": float(v[0]), "g1": g1, "g2": g2, "g3": g3, "g4": g4, "g5": g5}
    heads = []
    for t in model.tables[1:1 + model.ntypes]:
        fx = np.zeros(t.values.size, np.uint8) if t.fixed is None else t.fixed
        heads.append({"type": "linear", "coeffs": [float(x) for x in t.values[:-1]],
                      "fixed": bool(np.all(fx[:-1])) if t.values.size > 1 else False,
                      "bias": float(t.values[-1]), "bias_fixed": bool(fx[-1])})
    out = {"model": "ml", "ntypes": model.ntypes, "descriptor": desc, "heads": heads}
    if len(model.tables) == 1 + 2 * model.ntypes:  # add_standardization (output_writer.cpp:155-168)
        S = descriptor_size(model)
        out["standardization"] = [{"mean": [float(x) for x in t.values[:S]],
                                   "inv_std": [float(x) for x in t.values[S:]]}
                                  for t in model.tables[1 + model.ntypes:]]
    return json.dumps(out, indent=1)


def _tersoff_json(t):
    d = {}
    for k, nm in enumerate(TERSOFF_FIELDS):
        lo = -math.inf if t.lower is None else float(t.lower[k])
        hi = math.inf if t.upper is None else float(t.upper[k])
        fx = False if t.fixed is None else bool(t.fixed[k])
        if nm == "omega" and fx and math.isinf(lo) and math.isinf(hi) and float(t.values[k]) == 1.0:
            continue  # the reader's default: ω = 1, fixed
        if math.isinf(lo) and math.isinf(hi) and not fx:
            d[nm] = float(t.values[k])
        else:
            d[nm] = {"value": float(t.values[k]), "fixed": fx,
                     **({} if math.isinf(lo) else {"min": lo}), **({} if math.isinf(hi) else {"max": hi})}
    return d


def write_model(model):
    """Model → force-model JSON text, lossless: analytic tables keep their
    closed forms and parameter specs (families pair, eam, adp, angular,
    stiweb, tersoff, and ml with an ACSF descriptor).  write_native samples
    every radial table instead, as the reference's writer does."""
    nt, fam = model.ntypes, model.family
    npair = nt * (nt + 1) // 2
    if fam in (FS_FAMILY_ACSF, FS_FAMILY_LMBTR):
        return _write_ml(model)
    if fam == FS_FAMILY_TERSOFF:
        return json.dumps({"model": "tersoff", "ntypes": nt,
                           "potentials": [_tersoff_json(t) for t in model.tables]}, indent=1)
    if fam == FS_FAMILY_SW:
        # write_native for stiweb (output_writer.cpp:125-135): SWParams per
        # pair, then the triplet λ array
        def entry(t, k):
            lo = -math.inf if t.lower is None else float(t.lower[k])
            hi = math.inf if t.upper is None else float(t.upper[k])
            fx = False if t.fixed is None else bool(t.fixed[k])
            if math.isinf(lo) and math.isinf(hi) and not fx:
                return float(t.values[k])
            return {"value": float(t.values[k]), "fixed": fx,
                    **({} if math.isinf(lo) else {"min": lo}), **({} if math.isinf(hi) else {"max": hi})}
        pots = [{nm: entry(t, k) for k, nm in enumerate(SW_FIELDS)} for t in model.tables[:npair]]
        lam = model.tables[npair]
        return json.dumps({"model": "stiweb", "ntypes": nt, "potentials": pots,
                           "lambda": [entry(lam, k) for k in range(lam.values.size)]}, indent=1)
    if fam not in TABLE_KEYS:
        raise FormatError("write_model: unsupported model family")
    out = {"model": NAME_OF[fam], "ntypes": nt}
    names = [g.name or f"g{i}" for i, g in enumerate(model.globals)]
    refs = {}
    for g, gname in zip(model.globals, names):
        for tk, slot in g.links:
            refs.setdefault(tk, {})[slot] = gname
    if model.globals:
        out["globals"] = {gname: {"value": float(g.value), "fixed": bool(g.fixed)}
                          for g, gname in zip(model.globals, names)}
    k = 0
    for key in TABLE_KEYS[fam]:
        n = npair if PER_PAIR[key] else nt
        tabs = model.tables[k:k + n]
        fmt = "analytic" if all(t.kind == FS_TABLE_ANALYTIC for t in tabs) else "tabulated"
        out[key] = {"format": fmt, "potentials": [_pot_json(t, refs.get(k + i)) for i, t in enumerate(tabs)]}
        k += n
    return json.dumps(out, indent=1)


# ---------------------------------------------------------------------------
# LAMMPS setfl

def read_setfl(path):
    """Single-element setfl → (Model, header) with makima tables on the file's
    grids: φ = (r·φ)/r on r_k = k·dr (k = 1…Nr−1), ρ on r_k (k = 0…Nr−1),
    F on ρ_k = k·dρ (k = 0…Nρ−1).  Layout: three comment lines, "1 El",
    "Nrho drho Nr dr rc", "Z mass a0 lattice", then F, ρ, r·φ."""
    with open(path) as f:
        lines = f.read().split("\n")
    if int(lines[3].split()[0]) != 1:
        raise FormatError("read_setfl: single-element files only")
    nrho, drho, nr, dr, rc = lines[4].split()
    nrho, nr, drho, dr, rc = int(nrho), int(nr), float(drho), float(dr), float(rc)
    vals = np.array([float(v) for ln in lines[6:] for v in ln.split()])
    if vals.size < nrho + 2 * nr:
        raise FormatError("read_setfl: file ends early")
    F, rho, rphi = vals[:nrho], vals[nrho:nrho + nr], vals[nrho + nr:nrho + 2 * nr]
    r = dr * np.arange(1, nr)
    model = Model(FS_FAMILY_EAM, 1, [Table.spline(dr, dr * (nr - 1), rphi[1:] / r),
                                     Table.spline(0.0, dr * (nr - 1), rho),
                                     Table.spline(0.0, drho * (nrho - 1), F)])
    header = dict(element=lines[3].split()[1], nrho=nrho, drho=drho, nr=nr, dr=dr, rc=rc)
    return model, header


# ---------------------------------------------------------------------------
# sampled writers (src/io/output_writer.cpp, src/io/write_model.cpp)

DEFAULT_KNOTS = 500  # kDefaultKnots, include/forcesmith/io/output_writer.hpp:19


def _span(t):
    """RadialPotential::span: the knot span of a spline, the gate span of an
    analytic form."""
    return float(t.rmin), float(t.rmax)


def _grid(t, nknots):
    lo, hi = _span(t)
    step = (hi - lo) / (nknots - 1)
    return lo, hi, lo + np.arange(nknots) * step


def _sampled(model, k, sample, nknots):
    """sample_one (output_writer.cpp:22-40): {rmin, rmax, knots} of table k
    on nknots uniform points of its span; a non-finite value is an error."""
    lo, hi, r = _grid(model.tables[k], nknots)
    v, _ = sample(k, r)
    bad = np.nonzero(~np.isfinite(v))[0]
    if bad.size:
        q = int(bad[0])
        raise FormatError(f"non-finite potential value ({v[q]}) at r={r[q]:.6f}; "
                          "cannot tabulate potential for output")
    return {"rmin": lo, "rmax": hi, "knots": [float(x) for x in v]}


def session_sampler(sess):
    """The sampler of a GpuSession holding the model: fs_gpu_tabulate."""
    return lambda k, r: sess.tabulate(k, r)


def write_native(model, sample, nknots=DEFAULT_KNOTS):
    """write_native (output_writer.cpp:42-119): every radial table sampled
    onto nknots knots.  A pair model is a bare potential section; EAM, ADP and
    angular models are {"model", "ntypes", <section>: …}; Stillinger–Weber,
    Tersoff and ACSF models carry their parameters as they are.
    sample(k, r) → (values, derivatives) of table k at the points r."""
    fam, nt = model.family, model.ntypes
    if fam in (FS_FAMILY_TERSOFF, FS_FAMILY_ACSF, FS_FAMILY_LMBTR, FS_FAMILY_SW):
        return write_model(model)
    if fam not in TABLE_KEYS:
        raise FormatError("write_native: unsupported model family")
    npair = nt * (nt + 1) // 2
    if fam == FS_FAMILY_PAIR:
        return json.dumps({"format": "tabulated",
                           "potentials": [_sampled(model, k, sample, nknots) for k in range(npair)]}, indent=2)
    out, k = {"model": NAME_OF[fam], "ntypes": nt}, 0
    for key in TABLE_KEYS[fam]:
        n = npair if PER_PAIR[key] else nt
        out[key] = {"format": "tabulated",
                    "potentials": [_sampled(model, k + i, sample, nknots) for i in range(n)]}
        k += n
    return json.dumps(out, indent=2)


def _g(x):
    """A double as a default-formatted C++ stream writes it (6 significant
    digits, %g style)."""
    return format(float(x), "g")


def write_lammps(model, sample):
    """write_lammps (output_writer.cpp:266-289), pair models: per pair table
    a "# pair potential k" / "POT_k" / "N 500 R lo hi" block, then one
    "index r φ(r) φ'(r)" line per knot."""
    if model.family != FS_FAMILY_PAIR:
        raise FormatError("write_lammps: pair models only")
    lines = []
    for k, t in enumerate(model.tables):
        lo, hi, r = _grid(t, DEFAULT_KNOTS)
        v, dv = sample(k, r)
        lines += [f"# pair potential {k}", f"POT_{k}", f"N {DEFAULT_KNOTS} R {_g(lo)} {_g(hi)}", ""]
        lines += [f"{q + 1} {_g(r[q])} {_g(v[q])} {_g(dv[q])}" for q in range(DEFAULT_KNOTS)]
        lines.append("")
    return "\n".join(lines) + "\n"


def write_imd(model, sample):
    """write_imd (output_writer.cpp:291-310), pair models: the "#F 3 n",
    "#T IMD", "#E" header, one "lo hi 500" line per table, then every
    table's 500 values, one per line."""
    if model.family != FS_FAMILY_PAIR:
        raise FormatError("write_imd: pair models only")
    lines = [f"#F 3 {len(model.tables)}", "#T IMD", "#E"]
    lines += [f"{_g(_span(t)[0])} {_g(_span(t)[1])} {DEFAULT_KNOTS}" for t in model.tables]
    for k, t in enumerate(model.tables):
        _, _, r = _grid(t, DEFAULT_KNOTS)
        lines += [_g(x) for x in sample(k, r)[0]]
    return "\n".join(lines) + "\n"


def write_model_file(model, path, fmt, sample):
    """write_model (src/io/write_model.cpp:22-55): "lammps" and "imd" for
    pair models, native JSON otherwise (another format for another family
    writes native JSON with a warning on stderr)."""
    import sys
    if model.family == FS_FAMILY_PAIR and fmt == "lammps":
        text = write_lammps(model, sample)
    elif model.family == FS_FAMILY_PAIR and fmt == "imd":
        text = write_imd(model, sample)
    else:
        if fmt != "native" and model.family != FS_FAMILY_PAIR:
            print(f"warning: '{fmt}' output unsupported for {NAME_OF.get(model.family, 'ml')}; "
                  "writing native JSON", file=sys.stderr)
        text = write_native(model, sample)
    with open(path, "w") as f:
        f.write(text if text.endswith("\n") else text + "\n")
