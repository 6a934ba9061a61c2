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
