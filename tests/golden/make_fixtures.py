"""Makes the golden fixtures under tests/golden/ from the reference CAPS core (oracle/_ref, built from the reference's
sources by oracle/Makefile). Run here, where the reference is; the fixtures are committed so the GPU tests need no
reference at run time.

Each fixture is one cell (force field + positions + cell) and a set of option cases, each with the reference's forces
and energy terms in FP64 (EnergyOptions::mixed = false, the parity path) and in the reference's own mixed precision
(its FP32 cluster kernel), for comparing error levels.

    python tests/golden/make_fixtures.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from caps_b200 import EnergyOptions, ForceField  # noqa: E402
from oracle import ref  # noqa: E402


def charged_lj_triclinic(seed: int = 7) -> tuple[ForceField, np.ndarray, np.ndarray]:
    """1100 charged LJ sites on a jittered lattice in a triclinic cell, three types, chains of ten with 1-2 and 1-3
    partners excluded and 1-4 partners as 1-4 pairs (the kind of cell tests/nbnxm_check.cpp checks against a direct
    27-image sum; this generator is my own)."""
    rng = np.random.default_rng(seed)
    a, b, c = np.array([24.0, 0, 0]), np.array([3.0, 22.0, 0]), np.array([-2.0, 4.0, 23.0])
    nx, ny, nz = 10, 10, 11
    frac = np.array([[(i + 0.5) / nx, (j + 0.5) / ny, (k + 0.5) / nz] for k in range(nz) for j in range(ny) for i in range(nx)])
    frac += rng.uniform(-0.12, 0.12, frac.shape) / np.array([nx, ny, nz])
    x = frac @ np.vstack([a, b, c])
    n = len(x)
    types = np.arange(n) % 3
    eps = np.array([0.10, 0.15, 0.07])
    sig = np.array([3.2, 3.5, 2.9])
    pe = np.sqrt(np.outer(eps, eps))
    ps = 0.5 * (sig[:, None] + sig[None, :])
    q = np.where(np.arange(n) % 2 == 0, 0.31, -0.31)
    excl = [[] for _ in range(n)]
    p14 = []
    for s in range(0, n, 10):
        for i in range(s, min(s + 10, n)):
            for d in (1, 2, 3):
                j = i + d
                if j < min(s + 10, n):
                    excl[i].append(j)
                    excl[j].append(i)
                    if d == 3:
                        p14.append((i, j))
    off = np.zeros(n + 1, np.uint32)
    lst = []
    for i in range(n):
        e = sorted(excl[i])
        lst += e
        off[i + 1] = len(lst)
    ff = ForceField(type_index=types, charge=q, mass=np.full(n, 12.0), pair_eps=pe, pair_sigma=ps, pair14_ij=np.array(p14),
                    lj14=0.5, coul14=0.5, excl_offset=off, excl_list=np.array(lst), element=np.full(n, 6))
    cell = np.concatenate([np.zeros(3), a, b, c])
    return ff, x, cell


def cases_for(kind: str) -> list[dict]:
    if kind == "ps_small":
        out = []
        for el in ("pme", "dsf"):
            for tail in (True, False):
                out.append(dict(cutoff=8.0, skin=2.0, electrostatics=el, tail=tail, pme_order=5))
        out.append(dict(cutoff=9.0, skin=2.0, coulomb=False, tail=True))
        return out
    if kind == "ps_medium":
        return [dict(cutoff=10.0, skin=2.0, electrostatics="pme", tail=True, pme_order=4, pme_spacing=1.0),
                dict(cutoff=12.0, skin=2.0, electrostatics="pme", tail=False, pme_order=5, pme_spacing=1.2),
                dict(cutoff=10.0, skin=1.0, electrostatics="dsf", tail=True)]
    if kind == "lj_triclinic":
        return [dict(cutoff=9.0, skin=1.5, electrostatics="pme", tail=True, pme_order=6, pme_spacing=0.8, ewald_rtol=1e-6),
                dict(cutoff=9.0, skin=1.5, electrostatics="dsf", tail=False)]
    if kind == "kg":
        return [dict(cutoff=2.0 ** (1 / 6), skin=0.4, coulomb=False, tail=False)]
    raise KeyError(kind)


def save(name: str, ff: ForceField, x: np.ndarray, cell: np.ndarray, kind: str):
    arrays = {"ff_" + k: (np.asarray(v) if not isinstance(v, (bool, float, int)) else np.asarray(v)) for k, v in ff.arrays().items()}
    arrays["x"] = x
    arrays["cell"] = cell
    cases = cases_for(kind)
    meta = []
    for k, c in enumerate(cases):
        for prec in ("double", "mixed"):
            o = EnergyOptions(**{**c, "precision": prec})
            t, f = ref.compute(ff, o, x, cell, threads=1)
            arrays[f"f_{k}_{prec}"] = f
            meta.append({"case": k, "precision": prec, "options": {**c, "precision": prec}, "terms": t})
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / f"{name}.npz", **arrays)
    print(f"{name}: {ff.natoms} atoms, {len(cases)} cases")


def main():
    if not ref.available():
        raise SystemExit("oracle/_ref/libcaps_ref.so is missing: make -C oracle")
    ff, x, cell, ex = ref.build_ps_gaff(3, 4, 0.4, 0.9, 3)   # tests/test_nbnxm.cpp:19-34's cell
    assert ex["unsupported"] == 0
    save("ps_small", ff, x, cell, "ps_small")
    ff, x, cell, ex = ref.build_ps_gaff(8, 16, 0.3, 1.0, 11)
    assert ex["unsupported"] == 0
    save("ps_medium", ff, x, cell, "ps_medium")
    ff, x, cell = charged_lj_triclinic()
    save("lj_triclinic", ff, x, cell, "lj_triclinic")
    ff, x, cell, ex = ref.build_kg(20, 25, 0.85, 5)
    save("kg", ff, x, cell, "kg")


if __name__ == "__main__":
    main()
