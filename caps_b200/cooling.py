"""Stepwise cooling at constant pressure over batched replicas.

The reference's run_cooling (core/src/mechanics.cpp:1381-1470) runs one structure through a temperature ladder: an
unsampled hold at the starting temperature, then a hold at each temperature (Bussi thermostat, the chosen barostat,
seed + k for the k-th rung); the density and potential energy are averaged over the last part of each hold's thermo
rows. Here every stage of the ladder advances all replicas at once through `run_batch` (one CUDA graph launch per plain
step for all of them): the replicas of a Tg scan that differ in their seed, or in their structure, each get their own
points.

The glass-transition fit of the points stays with the caller, as it is host analysis and not part of the device path:
run_cooling takes it as a callable, fit(T, y, options) -> dict. CAPS passes its own fit_bilinear / fit_two_ranges
(core/src/mechanics.cpp:1218, 1310); without one the result's "fit" is None.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from .engine import DynamicsOptions, EnergyOptions, run_batch


@dataclass
class CoolingOptions:
    """caps::CoolingOptions (core/include/caps/mechanics.hpp:326-347), without the checkpoint and callback members."""
    energy: EnergyOptions = field(default_factory=EnergyOptions)
    t_start: float = 500.0
    t_end: float = 200.0
    t_step: float = 20.0          # K
    ps_per_step: float = 100.0    # hold at each temperature
    equilibrate_ps: float = -1.0  # unsampled hold at t_start first; -1: one hold
    average_from: float = 0.5     # fraction of each hold's rows left out of the averages
    dt: float = 1.0
    tau_t: float = 100.0
    tau_p: float = 1000.0
    pressure: float = 1.0
    compressibility: float = 4.5e-5
    barostat: str = "c-rescale"
    seed: int = 1
    new_velocities: bool = False
    property: int = 0             # Tg from 0 the specific volume, 1 the potential energy per atom
    fit: int = 0                  # for the caller's fit: 0 continuous two-line fit, 1 two ranges
    glassy_max: float = 0.0
    rubbery_min: float = 0.0

    def temperatures(self) -> list[float]:
        """The ladder, as mechanics.cpp:1386-1388 steps it."""
        if self.t_step <= 0 or self.ps_per_step <= 0:
            raise ValueError("temperature step and hold time must be positive")
        d = -1.0 if self.t_end < self.t_start else 1.0
        out, t = [], self.t_start
        while d * (t - self.t_end) <= 1e-9:
            out.append(t)
            t += d * self.t_step
        return out

    def hold_steps(self) -> int:
        return int(round_half_away(self.ps_per_step * 1000 / self.dt))

    def equilibration_steps(self) -> int:
        eq = self.ps_per_step if self.equilibrate_ps < 0 else self.equilibrate_ps
        return int(round_half_away(eq * 1000 / self.dt)) if eq > 0 else 0

    def _dyn(self, steps: int, temperature: float, seed: int, new_velocities: bool, thermo_every: int, offset: int) -> DynamicsOptions:
        return DynamicsOptions(dt=self.dt, steps=steps, temperature=temperature, thermostat="bussi", tau_t=self.tau_t, barostat=self.barostat,
                               pressure=self.pressure, tau_p=self.tau_p, compressibility=self.compressibility, seed=seed,
                               new_velocities=new_velocities, thermo_every=thermo_every, frame_every=0, step_offset=offset, energy=self.energy)


def round_half_away(v: float) -> float:
    """std::llround: halves away from zero."""
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


def hold_point(temperature: float, rows: list[dict], average_from: float) -> dict:
    """One temperature's point (mechanics.cpp:1440-1462): density and potential averaged over the rows from index
    average_from x len(rows) on, the density's standard error from five blocks of those rows."""
    first = int(average_from * len(rows))
    dens = [r["density"] for r in rows[first:]]
    pot = [r["potential"] for r in rows[first:]]
    p = {"temperature": temperature, "density": sum(dens) / max(1, len(dens)), "potential": sum(pot) / max(1, len(pot)),
         "density_err": 0.0}
    nb = min(5, len(dens))
    if nb >= 2:
        bm = []
        for b in range(nb):
            blk = dens[b * len(dens) // nb:(b + 1) * len(dens) // nb]
            bm.append(sum(blk) / max(1, len(blk)))
        v = sum((x - p["density"]) ** 2 for x in bm)
        p["density_err"] = math.sqrt(v / (nb - 1) / nb)
    p["specific_volume"] = 1 / p["density"] if p["density"] > 0 else 0.0
    return p


def run_cooling(evaluators: list, xs: list, cells: list, opts: list, vs: list | None = None,
                fit: Callable[[list, list, CoolingOptions], dict] | None = None) -> list[dict]:
    """run_cooling for every replica at once: one Evaluator, structure (x, cell) and CoolingOptions per replica. The
    options may differ in seed, pressure, barostat, thermostat coupling, property and fit, but not in the ladder (start,
    end, step, hold, equilibration, dt), since the replicas advance in lock step. Returns one result per replica:
    {points, fit, fitted, thermo, x, v, cell, method}; "fitted" is the property the fit reads (specific volume, or
    potential energy per atom) per point, and "fit" is fit(temperatures, fitted, options) of the caller's fit, or None.
    Replaces calling run_cooling (core/src/mechanics.cpp:1381) once per replica."""
    R = len(evaluators)
    if not (len(xs) == len(cells) == len(opts) == R) or R == 0:
        raise ValueError("run_cooling: one structure and one CoolingOptions per evaluator")
    sched = {(o.t_start, o.t_end, o.t_step, o.ps_per_step, o.equilibrate_ps, o.dt) for o in opts}
    if len(sched) != 1:
        raise ValueError("run_cooling: the replicas must share the temperature ladder, hold times and dt")
    o0 = opts[0]
    temps = o0.temperatures()
    steps = o0.hold_steps()
    eq = o0.equilibration_steps()
    xs = [np.asarray(x, dtype=np.float64).reshape(-1, 3).copy() for x in xs]
    cells = [np.asarray(c, dtype=np.float64).copy() for c in cells]
    vs = [None] * R if vs is None else [None if v is None else np.asarray(v, dtype=np.float64).reshape(-1, 3).copy() for v in vs]
    first_v = [o.new_velocities for o in opts]
    offset = 0
    thermo = [[] for _ in range(R)]
    points = [[] for _ in range(R)]

    def stage(dyn: list[DynamicsOptions]) -> list[dict]:
        if R == 1:
            out = [evaluators[0].run(xs[0], cells[0], dyn[0], v=vs[0])]
        else:
            out = run_batch(evaluators, xs, cells, dyn, vs)
        for r in range(R):
            xs[r], vs[r], cells[r] = out[r]["x"], out[r]["v"], out[r]["cell"]
        return out

    if eq > 0:
        dyn = [o._dyn(eq, o.t_start, o.seed + 1000, first_v[r], max(1, eq // 50), 0) for r, o in enumerate(opts)]
        stage(dyn)
        offset += eq
        first_v = [False] * R
    for k, t in enumerate(temps):
        dyn = [o._dyn(steps, t, o.seed + k, k == 0 and first_v[r], max(1, steps // 200), offset) for r, o in enumerate(opts)]
        out = stage(dyn)
        offset += steps
        for r in range(R):
            rows = out[r]["thermo"]
            thermo[r].extend(rows)
            points[r].append(hold_point(t, rows, opts[r].average_from))
    results = []
    for r, o in enumerate(opts):
        natoms = max(1, xs[r].shape[0])
        T = [p["temperature"] for p in points[r]]
        y = [p["potential"] / natoms if o.property == 1 else p["specific_volume"] for p in points[r]]
        result_fit = fit(T, y, o) if fit is not None else None
        what = "potential energy per atom" if o.property == 1 else "specific volume"
        how = "two lines through the glassy and the rubbery range" if o.fit == 1 else "a continuous two-line fit"
        method = (f"stepwise cooling {o.t_start:g} -> {o.t_end:g} K in {o.t_step:g} K steps of {o.ps_per_step:g} ps after "
                  f"{eq * o.dt / 1000:g} ps at {o.t_start:g} K ({o.barostat}, {o.pressure:g} atm); averages over the last "
                  f"{100 * (1 - o.average_from):g} % of each hold; Tg from {how} of {what}")
        results.append({"points": points[r], "fit": result_fit, "fitted": y, "thermo": thermo[r], "x": xs[r], "v": vs[r], "cell": cells[r],
                        "method": method})
    return results
