"""Makes the starting structure of the 32,000-atom polystyrene PME melt benchmark: caps_b200/data/ps32k_start.npz.

The cell is grown by caps_b200.systems.polystyrene_melt (40 chains x 50 repeat units, 1.04 g/cm^3, seed 1); the overlaps a
dense growth leaves are pushed off on the device (FP64, Langevin 500 K, the LJ force cap raised 5 -> 20 -> 100 -> 500
kcal/mol/Å as the reference's relax push-off does, Coulomb off, then on), then the melt is equilibrated with the
benchmark's own settings (mixed precision, SHAKE on C-H, Nose-Hoover 500 K, 1 fs) for `--ps` picoseconds. Positions and
velocities are stored in float32 (a starting point, not a result); the force field is rebuilt from the seed.

    python caps_b200/data/make_ps32k.py [--ps 5] [--out caps_b200/data/ps32k_start.npz]
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from caps_b200 import DynamicsOptions, EnergyOptions, Evaluator  # noqa: E402
from caps_b200.systems import polystyrene_melt  # noqa: E402

BENCH_ENERGY = dict(cutoff=12.0, skin=2.0, electrostatics="pme", ewald_rtol=1e-5, pme_spacing=1.0, pme_order=4, tail=True)


def push_off(ff, x, cell, log=print):
    for cap, coul in ((5.0, False), (20.0, False), (100.0, False), (500.0, False), (500.0, True)):
        eo = EnergyOptions(**{**BENCH_ENERGY, "coulomb": coul, "precision": "double", "force_cap": cap})
        o = DynamicsOptions(dt=0.5, steps=600, temperature=500.0, thermostat="langevin", tau_t=20.0, thermo_every=600, seed=7, energy=eo,
                            new_velocities=True)
        ev = Evaluator(ff, eo)
        out = ev.run(x, cell, o)
        x = out["x"]
        log(f"push-off cap {cap:6.0f} coulomb {coul}: T {out['thermo'][-1]['temperature']:.0f} K, "
            f"E {out['thermo'][-1]['potential']:.0f} kcal/mol")
        ev.close()
    return x


def equilibrate(ff, x, cell, ps: float, log=print):
    eo = EnergyOptions(**{**BENCH_ENERGY, "precision": "mixed"})
    o = DynamicsOptions(dt=1.0, steps=int(ps * 1000), temperature=500.0, thermostat="nose-hoover", tau_t=100.0, thermo_every=1000,
                        constraints="h-bonds", seed=11, energy=eo, new_velocities=True)
    ev = Evaluator(ff, eo)
    out = ev.run(x, cell, o)
    for r in out["thermo"]:
        log(f"  equilibrate step {r['step']:6d}: T {r['temperature']:.1f} K, E {r['potential']:.1f}, conserved {r['conserved']:.1f}")
    return out["x"], out["v"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ps", type=float, default=5.0)
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent / "ps32k_start.npz"))
    a = ap.parse_args()
    t0 = time.time()
    ff, x, cell = polystyrene_melt(40, 50, 1.04, seed=1)
    print(f"grown {ff.natoms} atoms in {time.time() - t0:.1f} s, box {cell[3]:.3f} Å")
    x = push_off(ff, x, cell)
    x, v = equilibrate(ff, x, cell, a.ps)
    np.savez_compressed(a.out, x=x.astype(np.float32), v=v.astype(np.float32), cell=cell)
    print(f"wrote {a.out} after {time.time() - t0:.1f} s")


if __name__ == "__main__":
    main()
