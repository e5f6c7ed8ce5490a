"""The Al fcc LM-fit fixture (tests/golden/al99_c1.npz, written by
tests/golden/make_al99.py) as a Dataset and the 15-knot start Model."""
import os

import numpy as np

from forcesmith_b200.abi import FS_FAMILY_EAM, Dataset, Model, Table

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "al99_c1.npz")


def load():
    z = np.load(PATH)
    ds = Dataset(z["natoms"], z["box9"], z["pos"], z["type"], z["forces"], z["energy"], z["stress9"])
    tabs = [Table.spline(float(lo), float(hi), z["start_knots"][k]) for k, (lo, hi) in enumerate(z["start_domains"])]
    return ds, Model(FS_FAMILY_EAM, 1, tabs), float(z["ideal_energy_per_atom"])
