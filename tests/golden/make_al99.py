"""Writes tests/golden/al99_c1.npz: the Al fcc LM-fit fixture.

Run in a checkout that has the Forcesmith sources beside it (it reads their
data/Al99.eam.alloy, a LAMMPS setfl table); the GPU tests use only the .npz.

  geometry  20 configurations of fcc Al, 3×3×3 conventional cells (108 atoms),
            a = 4.05 Å, Gaussian displacements σ = 0.10 Å, isotropic box
            strain U[0.97, 1.03] (forcesmith_b200.synth.fcc, seed 20261203)
  labels    forces, energies and stresses of the Al99 potential evaluated by
            the FP64 oracle, with makima splines on the file's own grids:
            φ = (rφ)/r on r_k = k·dr (k = 1…Nr−1), ρ on r_k (k = 0…Nr−1),
            F on ρ_k = k·dρ (k = 0…Nρ−1)
  start     three 15-knot splines on φ: [dr, rc], ρ: [0, rc],
            F: [0, (Nρ−1)·dρ], knot values read off the label splines and
            multiplied by U[0.95, 1.05] (seed 7)

setfl layout (LAMMPS): three comment lines; "1 Al"; "Nrho drho Nr dr rc";
"Z mass a0 lattice"; then F(ρ)[Nrho], ρ(r)[Nr], r·φ(r)[Nr].
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from forcesmith_b200 import synth  # noqa: E402
from forcesmith_b200.io import read_setfl  # noqa: E402
from oracle import api as O  # noqa: E402

# The reference's data/Al99.eam.alloy; give its path in AL99_SETFL, or the
# Forcesmith source tree in FORCESMITH_SRC.
SETFL = os.environ.get("AL99_SETFL") or os.path.join(os.environ.get("FORCESMITH_SRC", ""), "data",
                                                      "Al99.eam.alloy")


def main():
    label, t = read_setfl(SETFL)
    nr, dr, nrho, drho = t["nr"], t["dr"], t["nrho"], t["drho"]
    phi, rho, F = (tb.values for tb in label.tables)
    ds = synth.fcc(20, 3, 4.05, 0.10, 0.97, 1.03, seed=20261203)
    o = O.Oracle()
    o.upload(ds.with_labels(np.zeros((ds.n_atoms, 3)), np.zeros(ds.n_cfg), np.zeros((ds.n_cfg, 9))))
    o.set_model(label)
    out = o.eval(1.0, 0.0, want=("forces", "energy", "stress"))
    # pin of the parse: the ideal crystal's energy per atom (published for this
    # potential: cohesive energy 3.36 eV at a0 = 4.05 Å)
    ideal = synth.fcc(1, 3, 4.05, 0.0, 1.0, 1.0, seed=1)
    oi = O.Oracle()
    oi.upload(ideal.with_labels(np.zeros((ideal.n_atoms, 3)), np.zeros(1), np.zeros((1, 9))))
    oi.set_model(label)
    e_ideal = float(oi.eval(1.0, 0.0, want=("energy",))["energy"][0]) / ideal.n_atoms
    # start model: 15 knots per table, read off the label splines, perturbed
    doms = [(dr, t["rc"]), (0.0, t["rc"]), (0.0, drho * (nrho - 1))]
    grids = [(dr * np.arange(1, nr), phi), (dr * np.arange(nr), rho), (drho * np.arange(nrho), F)]
    rng = synth.uniform(45, 0.95, 1.05, 7)
    knots = []
    for k, ((lo, hi), (x, y)) in enumerate(zip(doms, grids)):
        xs = np.linspace(lo, hi, 15)
        v = np.array([O.spline_eval(x, y, float(xx))[0] for xx in xs])
        knots.append(v * rng[15 * k:15 * (k + 1)])
    np.savez_compressed(os.path.join(HERE, "al99_c1.npz"), natoms=ds.natoms, box9=ds.box9, pos=ds.pos,
                        type=ds.type, forces=out["forces"], energy=out["energy"], stress9=out["stress"],
                        start_knots=np.stack(knots), start_domains=np.array(doms), ideal_energy_per_atom=e_ideal)
    print("wrote al99_c1.npz", ds.n_atoms, "atoms; ideal-crystal energy per atom", e_ideal)


if __name__ == "__main__":
    main()
