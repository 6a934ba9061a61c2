"""Loads the golden fixtures of tests/golden (made by tests/golden/make_fixtures.py from the reference core)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from caps_b200 import EnergyOptions, ForceField

GOLDEN = Path(__file__).resolve().parent / "golden"
NAMES = ["ps_small", "ps_medium", "lj_triclinic", "kg"]


class Fixture:
    def __init__(self, name: str):
        z = np.load(GOLDEN / f"{name}.npz")
        self.name = name
        self.ff = ForceField.from_arrays({k[3:]: z[k] for k in z.files if k.startswith("ff_")})
        self.x = z["x"]
        self.cell = z["cell"]
        self.meta = json.loads(bytes(z["meta"]).decode())
        self.forces = {(m["case"], m["precision"]): z[f"f_{m['case']}_{m['precision']}"] for m in self.meta}

    def cases(self):
        """(case index, options dict) for each option case."""
        seen = {}
        for m in self.meta:
            seen.setdefault(m["case"], {k: v for k, v in m["options"].items() if k != "precision"})
        return sorted(seen.items())

    def options(self, case: int, precision: str) -> EnergyOptions:
        return EnergyOptions(**{**dict(self.cases())[case], "precision": precision})

    def terms(self, case: int, precision: str) -> dict:
        for m in self.meta:
            if m["case"] == case and m["precision"] == precision:
                return m["terms"]
        raise KeyError((case, precision))


def load(name: str) -> Fixture:
    return Fixture(name)


def rel_rms(f, ref) -> float:
    """RMS force error relative to the RMS force (the reference's own measure, tests/test_nbnxm.cpp:57-60)."""
    f, ref = np.asarray(f).reshape(-1), np.asarray(ref).reshape(-1)
    return float(np.sqrt(np.mean((f - ref) ** 2) / np.mean(ref ** 2)))


def rel_max(f, ref) -> float:
    """Largest component error relative to the RMS force."""
    f, ref = np.asarray(f).reshape(-1), np.asarray(ref).reshape(-1)
    return float(np.max(np.abs(f - ref)) / np.sqrt(np.mean(ref ** 2)))


# Trajectory writer cases: seeded frames in cells of every shape the writers treat apart (LAMMPS's own form, a cell
# needing the rotation, a left-handed one, an orthogonal one, none).
TRAJ_CELLS = {
    "lammps_form": [1.0, 2.0, 3.0, 20.0, 0.0, 0.0, 1.5, 18.0, 0.0, -2.0, 3.0, 21.0],
    "rotated": [0.5, -0.2, 0.1, 20.0, 0.3, -0.4, 1.5, 18.0, 0.7, -2.0, 3.0, 21.0],
    "orthogonal": [0.0, 0.0, 0.0, 20.0, 0.0, 0.0, 0.0, 18.0, 0.0, 0.0, 0.0, 21.0],
    "left_handed": [0.0, 0.0, 0.0, 20.0, 0.0, 0.0, 0.0, 18.0, 0.0, 0.0, 0.0, -21.0],
    "no_cell": [0.0] * 12,
}
TRAJ_FORMATS = ["lammpstrj", "dcd", "trr"]


def trajectory_case(cell_name: str, natoms: int = 37, nframes: int = 5, seed: int = 11):
    """(ids, mols, types, frames [(x, cell, step)]) of one writer case; the same numbers on every machine."""
    rng = np.random.default_rng(seed)
    ids = np.arange(1, natoms + 1, dtype=np.int64) * 2 + 5
    mols = np.arange(natoms, dtype=np.int64) // 4 + 1
    types = (np.arange(natoms, dtype=np.int32) % 5) + 1
    cell0 = np.asarray(TRAJ_CELLS[cell_name], dtype=np.float64)
    frames = []
    for k in range(nframes):
        x = rng.normal(0.0, 6.0, size=(natoms, 3)) + 10.0
        frames.append((x, cell0 * (1.0 + 0.003 * k), 1000 + 250 * k))
    return ids, mols, types, frames


def ps32k():
    """The 32,000-atom polystyrene PME melt of the benchmark (40 chains x 50 units x 16 atoms at 1.04 g/cm3): its force
    field from caps_b200.systems and the committed equilibrated start structure. (ff, x, v, cell)"""
    from caps_b200.systems import polystyrene_melt
    z = np.load(Path(__file__).resolve().parent.parent / "caps_b200" / "data" / "ps32k_start.npz")
    ff, _, _ = polystyrene_melt(40, 50, 1.04, seed=1, grow=False)
    return ff, z["x"].astype(np.float64), z["v"].astype(np.float64), z["cell"].astype(np.float64)


def ps32k_options(precision: str, tail: bool = True) -> EnergyOptions:
    """The benchmark's energy options: r_c 12 Å + 2 Å skin, PME rtol 1e-5, 1 Å spacing, order 4."""
    return EnergyOptions(cutoff=12.0, skin=2.0, electrostatics="pme", ewald_rtol=1e-5, pme_spacing=1.0, pme_order=4, tail=tail,
                         precision=precision)
