"""The evaluate path: one residual evaluation of every configuration and the
report of the reference's `--evaluate` option (src/cli/evaluate_report.cpp:21-83;
Forcesmith::evaluate_all, src/api/forcesmith.cpp:587-614).

Per configuration: calculated and reference energy, stress in Voigt order
00, 11, 22, 01, 02, 12, per-atom calculated and reference forces, the clamp
penalty `limit`, and `sumsq`:
    Σ‖F_calc − F_ref‖² + (w_e ΔE)² + [w_s > 0] Σ (w_s Δσ)² + limit²,
which summed over configurations (`total_sumsq`) is the objective ‖F‖² of the
residual vector.
"""
from __future__ import annotations

import json

import numpy as np

VOIGT6 = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))


def evaluate_report(sess, ds, w_e=1.0, w_s=0.0, names=None):
    """Report dict for the dataset `ds` already uploaded to `sess` (a
    GpuSession, or any session with the same `eval`)."""
    out = sess.eval(w_e, w_s, want=("forces", "energy", "stress", "limit", "obj"))
    fc, en, st, lim = out["forces"], out["energy"], out["stress"], out["limit"]
    report = {"energy_weight": w_e, "stress_weight": w_s, "nconf": int(ds.n_cfg), "configs": []}
    total, a0 = 0.0, 0
    for c in range(ds.n_cfg):
        n = int(ds.natoms[c])
        cf, rf = fc[a0:a0 + n], ds.ref_force[a0:a0 + n]
        csq = float(np.sum((cf - rf) ** 2))
        de = w_e * (en[c] - ds.ref_energy[c])
        csq += de * de
        s, sr = st[c].reshape(3, 3), np.asarray(ds.ref_stress9[c]).reshape(3, 3)
        if w_s > 0.0:
            csq += sum((w_s * (s[i, j] - sr[i, j])) ** 2 for i, j in VOIGT6)
        csq += lim[c] * lim[c]
        total += csq
        report["configs"].append({
            "index": c, "name": "" if names is None else names[c], "natoms": n,
            "calc_energy": float(en[c]), "ref_energy": float(ds.ref_energy[c]),
            "calc_stress": [float(s[i, j]) for i, j in VOIGT6],
            "ref_stress": [float(sr[i, j]) for i, j in VOIGT6],
            "atoms": [{"calc_force": [float(v) for v in cf[k]], "ref_force": [float(v) for v in rf[k]]}
                      for k in range(n)],
            "limit": float(lim[c]), "sumsq": csq})
        a0 += n
    report["total_sumsq"] = total
    return report


def write_evaluate_report(path, sess, ds, w_e=1.0, w_s=0.0, names=None):
    rep = evaluate_report(sess, ds, w_e, w_s, names)
    with open(path, "w") as f:
        f.write(json.dumps(rep, indent=2) + "\n")
    return rep
