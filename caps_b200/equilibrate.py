"""Equilibration protocols as chained dynamics stages on persistent engines, over batched replicas.

The reference's equilibrate (core/src/equilibrate.cpp:199-357) runs a list of stages (NVT / NPT / NVE, a duration, a
temperature or a ramp, a pressure, an optional LJ force cap) one after another on one structure, each stage a
run_dynamics call that builds a new Evaluator. Here each replica keeps one device engine (its force field uploaded
once) for every stage, and every stage advances all replicas at once through `run_batch` (the 21-step protocol over
seeds, for instance). The protocols (Larsen et al. 21-step, annealing, push-off) and the plain-text protocol format are
the reference's (equilibrate.cpp:43-197). The convergence blocks that may follow the stages (until_converged) are not
run on the device: they need the reference's chain-shape analyses between blocks.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np

from .engine import DynamicsOptions, run_batch

BAR_TO_ATM = 1.0 / 1.01325


@dataclass
class Stage:
    """caps::Stage (core/include/caps/equilibrate.hpp:15-22)."""
    label: str = ""
    ensemble: str = "nvt"          # "nvt" | "npt" | "nve"
    ps: float = 10.0
    t_start: float = 300.0
    t_end: float = -1.0            # >= 0 ramps the thermostat target
    pressure: float = 1.0          # atm, NPT only
    force_cap: float = 0.0         # kcal/mol/Å; > 0 caps the LJ forces (push-off; FP64 engines only)


@dataclass
class ProtocolParams:
    """caps::ProtocolParams (equilibrate.hpp:24-38)."""
    t_final: float = 300.0
    t_max: float = 600.0
    p_final: float = 1.0
    p_max: float = 49346.2
    time_scale: float = 1.0
    cycles: int = 3
    t_low: float = 300.0
    t_high: float = 600.0
    ramp_ps: float = 50.0
    hold_ps: float = 50.0
    caps: list = field(default_factory=lambda: [5.0, 10.0, 20.0, 50.0, 100.0, 200.0, 500.0])
    cap_ps: float = 5.0


def _nvt(label, ps, t):
    return Stage(label=label, ensemble="nvt", ps=ps, t_start=t)


def _npt(label, ps, t, p):
    return Stage(label=label, ensemble="npt", ps=ps, t_start=t, pressure=p)


def larsen21(p: ProtocolParams) -> list[Stage]:
    """The 21-step compression and decompression protocol (Larsen, Lin, Hart and Colina, Macromolecules 44, 6944
    (2011), Table 1), as equilibrate.cpp:43-56 lays it out."""
    tm, tf, pm = p.t_max, p.t_final, p.p_max
    s = [_nvt("1 · heat", 50, tm), _nvt("2 · cool", 50, tf), _npt("3 · compress 0.02 Pmax", 50, tf, 0.02 * pm),
         _nvt("4 · heat", 50, tm), _nvt("5 · cool", 100, tf), _npt("6 · compress 0.6 Pmax", 50, tf, 0.6 * pm),
         _nvt("7 · heat", 50, tm), _nvt("8 · cool", 100, tf), _npt("9 · compress Pmax", 50, tf, pm),
         _nvt("10 · heat", 50, tm), _nvt("11 · cool", 100, tf), _npt("12 · decompress 0.5 Pmax", 5, tf, 0.5 * pm),
         _nvt("13 · heat", 5, tm), _nvt("14 · cool", 10, tf), _npt("15 · decompress 0.1 Pmax", 5, tf, 0.1 * pm),
         _nvt("16 · heat", 5, tm), _nvt("17 · cool", 10, tf), _npt("18 · decompress 0.01 Pmax", 5, tf, 0.01 * pm),
         _nvt("19 · heat", 5, tm), _nvt("20 · cool", 10, tf), _npt("21 · final", 800, tf, p.p_final)]
    for st in s:
        st.ps *= p.time_scale
    return s


def annealing(p: ProtocolParams) -> list[Stage]:
    """NPT ramps between t_low and t_high with holds, `cycles` times (equilibrate.cpp:58-74)."""
    k = p.time_scale
    s = [_npt("settle", p.hold_ps * k, p.t_low, p.p_final)]
    for c in range(1, p.cycles + 1):
        up = _npt(f"cycle {c} · heat", p.ramp_ps * k, p.t_low, p.p_final)
        up.t_end = p.t_high
        down = _npt(f"cycle {c} · cool", p.ramp_ps * k, p.t_high, p.p_final)
        down.t_end = p.t_low
        s += [up, _npt(f"cycle {c} · hold", p.hold_ps * k, p.t_high, p.p_final), down, _npt(f"cycle {c} · hold", p.hold_ps * k, p.t_low, p.p_final)]
    return s


def pushoff(p: ProtocolParams) -> list[Stage]:
    """NVT with the LJ forces capped at increasing values, then uncapped NVT and NPT (equilibrate.cpp:76-87)."""
    k = p.time_scale
    s = []
    for cap in p.caps:
        st = _nvt(f"push-off · cap {cap:g}", p.cap_ps * k, p.t_final)
        st.force_cap = cap
        s.append(st)
    return s + [_nvt("uncapped", 20 * k, p.t_final), _npt("NPT", 50 * k, p.t_final, p.p_final)]


def protocol_by_name(name: str, p: ProtocolParams) -> list[Stage]:
    if not p.time_scale > 0:
        raise ValueError(f"the time scale must be above 0 (got {p.time_scale})")
    if not (p.ramp_ps >= 0 and p.hold_ps >= 0 and p.cap_ps >= 0):
        raise ValueError("stage lengths (ramp, hold, push-off) must be 0 ps or more")
    if p.cycles < 0:
        raise ValueError("the number of annealing cycles must be 0 or more")
    if name in ("larsen21", "21-step"):
        return larsen21(p)
    if name in ("annealing", "anneal"):
        return annealing(p)
    if name in ("pushoff", "push-off"):
        return pushoff(p)
    raise ValueError(f"unknown protocol '{name}' (larsen21, annealing, pushoff)")


def parse_protocol(text: str) -> list[Stage]:
    """Plain-text protocols, one stage per line (equilibrate.cpp:100-164): 'nvt 50 ps T 600', 'npt 50 ps T 300 P 987 atm'
    (or bar), 'nvt 20 ps T 300 to 600', 'nvt 5 ps T 300 cap 20', 'nve 10 ps'; '#' starts the stage's label."""
    out = []
    for lineno, line in enumerate(text.split("\n"), 1):
        label = ""
        if "#" in line:
            h = line.index("#")
            label = line[h + 1:].lstrip(" ").rstrip(" \r")
            line = line[:h]
        t = [w.lower() for w in line.split()]
        if not t:
            continue

        def bad(why):
            return ValueError(f"protocol line {lineno}: {why}")

        def num(i):
            if i >= len(t):
                raise bad(f"a number is missing after '{t[i - 1]}'")
            try:
                return float(t[i])
            except ValueError:
                raise bad(f"'{t[i]}' is not a number") from None

        if t[0] not in ("nvt", "npt", "nve"):
            raise bad(f"starts with '{t[0]}'; expected nvt, npt or nve")
        s = Stage(ensemble=t[0])
        have_time = have_p = False
        i = 1
        while i < len(t):
            if i + 1 < len(t) and t[i + 1] in ("ps", "ns", "fs"):
                v = num(i)
                s.ps = v * 1000 if t[i + 1] == "ns" else v / 1000 if t[i + 1] == "fs" else v
                have_time = True
                i += 1
            elif t[i] == "t":
                i += 1
                s.t_start = num(i)
                if i + 1 < len(t) and t[i + 1] in ("to", "->"):
                    i += 2
                    s.t_end = num(i)
            elif t[i] == "p":
                i += 1
                s.pressure = num(i)
                have_p = True
                if i + 1 < len(t) and t[i + 1] in ("bar", "atm"):
                    if t[i + 1] == "bar":
                        s.pressure *= BAR_TO_ATM
                    i += 1
            elif t[i] == "cap":
                i += 1
                s.force_cap = num(i)
            else:
                raise bad(f"does not understand '{t[i]}'")
            i += 1
        if not have_time or s.ps <= 0:
            raise bad("needs a duration, e.g. '50 ps'")
        if s.ensemble == "npt" and not have_p:
            raise bad("npt needs a pressure, e.g. 'P 1 atm'")
        s.label = label if label else f"{len(out) + 1} · {t[0]}"
        out.append(s)
    if not out:
        raise ValueError("the protocol has no stages")
    return out


def protocol_ps(stages: list[Stage]) -> float:
    return sum(s.ps for s in stages)


@dataclass
class EquilibrateOptions:
    """caps::EquilibrateOptions (equilibrate.hpp:70-85) without the convergence blocks, frames and checkpoints: the stages
    and the base dynamics options (dt, thermostat / barostat kinds and times, seed, energy options)."""
    stages: list = field(default_factory=list)
    md: DynamicsOptions = field(default_factory=DynamicsOptions)
    thermo_ps: float = 0.5        # a thermo row this often; 0: about 200 rows per stage (every 10 steps to 0.5 ps)

    def stage_steps(self, st: Stage) -> int:
        return max(1, int(_llround(st.ps * 1000.0 / self.md.dt)))

    def stage_options(self, st: Stage, k: int, offset: int) -> DynamicsOptions:
        """The run_dynamics options of stage k (equilibrate.cpp:210-236)."""
        md, dt = self.md, self.md.dt
        thermostat = "none" if st.ensemble == "nve" else ("bussi" if md.thermostat.lower() in ("none", "nve") else md.thermostat)
        barostat = ("c-rescale" if md.barostat.lower() == "none" else md.barostat) if st.ensemble == "npt" else "none"
        tps = self.thermo_ps if self.thermo_ps > 0 else min(max(st.ps / 200.0, 10.0 * dt / 1000.0), 0.5)
        energy = replace(md.energy, force_cap=st.force_cap)
        return replace(md, steps=self.stage_steps(st), temperature=st.t_start, temperature_end=st.t_end, thermostat=thermostat,
                       barostat=barostat, pressure=st.pressure, energy=energy, seed=md.seed + 1000003 * k, step_offset=offset,
                       thermo_every=max(1, int(_llround(tps * 1000.0 / dt))), frame_every=0, new_velocities=False)


def _llround(v: float) -> float:
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


def equilibrate(evaluators: list, xs: list, cells: list, opts: list, vs: list | None = None) -> list[dict]:
    """equilibrate for every replica at once: one Evaluator (its engine kept for every stage), structure and
    EquilibrateOptions per replica; the replicas may differ in seed, thermostat and barostat settings and pressures of
    their stages, not in the stages' lengths or dt. Returns per replica {stages (label, ps, temperature, pressure,
    density, potential averaged over each stage's second half, density_end), thermo (a stage's first row, which repeats
    the previous stage's last, left out), x, v, cell, ps}. Replaces calling equilibrate (core/src/equilibrate.cpp:199)
    once per replica."""
    R = len(evaluators)
    if not (len(xs) == len(cells) == len(opts) == R) or R == 0:
        raise ValueError("equilibrate: one structure and one EquilibrateOptions per evaluator")
    if any(not o.stages for o in opts):
        raise ValueError("the protocol has no stages")
    lengths = {(o.md.dt, tuple(o.stage_steps(st) for st in o.stages)) for o in opts}
    if len(lengths) != 1:
        raise ValueError("equilibrate: the replicas must share dt and the stages' lengths")
    xs = [np.asarray(x, dtype=np.float64).reshape(-1, 3).copy() for x in xs]
    cells = [np.asarray(c, dtype=np.float64).copy() for c in cells]
    vs = [None] * R if vs is None else [None if v is None else np.asarray(v, dtype=np.float64).reshape(-1, 3).copy() for v in vs]
    masses = [float(np.sum(ev.ff.mass)) for ev in evaluators]
    thermo = [[] for _ in range(R)]
    summaries = [[] for _ in range(R)]
    offset = 0
    for k in range(len(opts[0].stages)):
        dyn = [o.stage_options(o.stages[k], k, offset) for o in opts]
        if R == 1:
            out = [evaluators[0].run(xs[0], cells[0], dyn[0], v=vs[0])]
        else:
            out = run_batch(evaluators, xs, cells, dyn, vs)
        for r in range(R):
            xs[r], vs[r], cells[r] = out[r]["x"], out[r]["v"], out[r]["cell"]
            first = len(thermo[r])
            for row in out[r]["thermo"]:
                if thermo[r] and thermo[r][-1]["step"] == row["step"]:
                    continue
                thermo[r].append(row)
            a = first + (len(thermo[r]) - first) // 2
            tail = thermo[r][a:]
            n = len(tail)
            st = opts[r].stages[k]
            summ = {"label": st.label, "ps": dyn[r].steps * dyn[r].dt / 1000.0}
            for key in ("temperature", "pressure", "density", "potential"):
                acc = 0.0
                for row in tail:
                    acc += row[key] / n
                summ[key] = acc
            vol = abs(float(np.linalg.det(np.asarray(cells[r][3:12]).reshape(3, 3))))
            summ["density_end"] = masses[r] / 6.02214076e23 / (vol * 1e-24)
            summaries[r].append(summ)
        offset += dyn[0].steps
    return [{"stages": summaries[r], "thermo": thermo[r], "x": xs[r], "v": vs[r], "cell": cells[r], "ps": offset * opts[r].md.dt / 1000.0}
            for r in range(R)]
