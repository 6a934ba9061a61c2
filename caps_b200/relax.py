"""Structure relaxation on one device engine: the reference's relax (core/src/relax.cpp:343-369) and its stage chain
relax_once (relax.cpp:371-700): push-off by dynamics with a ramped LJ force cap, push-off minimisations under rising
caps, compression stage by stage, the final minimisation, and box relaxation towards a pressure (isotropic, or axis by
axis), then the linear-angle kicks of relax (kick_linear_angles, relax.cpp:304-338). Every stage runs on the same
engine: the force field is uploaded once, and a stage changes only the engine's options (a force cap, Coulomb off), as
the reference changes its evaluator's (Evaluator::set_options).

Under a force cap the reference evaluates on its FP64 path whatever the precision asked (field.cpp:845); so do the
capped stages here. The host arithmetic (stage plans, affine scaling, the secant iteration on the volume, the kicks'
random stream) follows the reference's, so an FP64 engine takes the reference's path.
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field

import numpy as np

from .engine import DynamicsOptions, EnergyOptions, FieldError, cell_array
from .minimise import (MinimiseOptions, cell_valid as _valid, cell_volume as _volume, cross3 as _cross, dot3 as _dot, max_force,
                       minimise, minimum_image, round_half_away as _round)

KNA = 6.02214076e23
KATM = 68568.415   # kcal/(mol Å³) -> atm


@dataclass
class RelaxOptions(MinimiseOptions):
    """caps::RelaxOptions (core/include/caps/relax.hpp:27-84) without the force field (the engine's), the cell-fit check
    and the callbacks."""
    energy: EnergyOptions = field(default_factory=EnergyOptions)
    pushoff: bool = True
    pushoff_caps: list = field(default_factory=lambda: [5.0, 20.0, 100.0, 500.0])   # kcal/mol/Å
    pushoff_ramp_ps: float = 0.0
    pushoff_cap: float = 0.0
    pushoff_temperature: float = 300.0
    pushoff_ramp_segments: int = 10
    target_density: float = 0.0      # g/cm³, 0: keep the cell
    compress_step: float = 0.06
    relax_box: bool = False
    pressure: float = 1.0            # atm
    pressure_tol: float = 100.0      # atm
    box_cycles: int = 40
    box_anisotropic: bool = False
    box_axes: tuple = (True, True, True)


# --- the reference's random stream, restated ------------------------------------------------------------------

class _MT64:
    """std::mt19937_64 (its parameters are fixed by the C++ standard)."""
    N, M = 312, 156

    def __init__(self, seed: int):
        mask = (1 << 64) - 1
        self.mt = [0] * self.N
        self.mt[0] = seed & mask
        for i in range(1, self.N):
            self.mt[i] = (6364136223846793005 * (self.mt[i - 1] ^ (self.mt[i - 1] >> 62)) + i) & mask
        self.i = self.N

    def __call__(self) -> int:
        mask, up, lo = (1 << 64) - 1, 0xFFFFFFFF80000000, 0x7FFFFFFF
        if self.i >= self.N:
            mt = self.mt
            for k in range(self.N):
                y = (mt[k] & up) | (mt[(k + 1) % self.N] & lo)
                mt[k] = mt[(k + self.M) % self.N] ^ (y >> 1) ^ (0xB5026F5AA96619E9 if y & 1 else 0)
            self.i = 0
        y = self.mt[self.i]
        self.i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & mask


class _Normal:
    """caps::Normal (core/include/caps/rng.hpp): Marsaglia's polar method on 53-bit uniforms, the second value kept."""

    def __init__(self):
        self.spare = None

    def __call__(self, g: _MT64) -> float:
        if self.spare is not None:
            s, self.spare = self.spare, None
            return s
        while True:
            u = 2 * ((g() >> 11) * 2.0 ** -53) - 1
            v = 2 * ((g() >> 11) * 2.0 ** -53) - 1
            q = u * u + v * v
            if not (q >= 1 or q == 0):
                break
        f = math.sqrt(-2 * math.log(q) / q)
        self.spare = v * f
        return u * f


def kick_linear_angles(x: np.ndarray, cell, ff, seed: int, min_deg: float = 172.0, fixed=None) -> int:
    """kick_linear_angles (relax.cpp:304-338): every angle centre with theta0 below 150 degrees held above min_deg moves
    0.15 Å perpendicular to the line of its two partners, in a direction from the seed's normal stream; x (N x 3) in
    place. Returns how many moved."""
    kdeg = math.pi / 180.0
    c = cell_array(cell)
    pos = x.reshape(-1, 3)

    def vec(a, b):
        return minimum_image(c, tuple(float(pos[a][k] - pos[b][k]) for k in range(3)))

    centres, ends = [], {}
    for (i, j, k), (_, th0) in zip(ff.angle_ijk.tolist(), ff.angle_kt_theta0.tolist()):
        if th0 >= 150.0 * kdeg:
            continue
        u, v = vec(i, j), vec(k, j)
        cs = _dot(u, v) / (math.sqrt(_dot(u, u)) * math.sqrt(_dot(v, v)))
        if cs > math.cos(min_deg * kdeg):
            continue
        if fixed is not None and len(fixed) == len(pos) and fixed[j]:
            continue
        if j not in ends:
            ends[j] = (i, k)
            centres.append(j)
    g, nd = _MT64(seed), _Normal()
    for j in sorted(centres):
        i, k = ends[j]
        axis = vec(k, i)
        na = max(1e-9, math.sqrt(_dot(axis, axis)))
        axis = tuple(q * (1.0 / na) for q in axis)
        r = (nd(g), nd(g), nd(g))
        dr = _dot(r, axis)
        r = tuple(r[m] - axis[m] * dr for m in range(3))
        n = math.sqrt(_dot(r, r))
        if n < 1e-9:
            continue
        for m in range(3):
            pos[j][m] = pos[j][m] + r[m] * (0.15 / n)
    return len(centres)


def _scale_affine(x: np.ndarray, c: np.ndarray, s: float):
    """scale_affine (relax.cpp:294-300): positions and cell about the cell origin."""
    p = x.reshape(-1, 3)
    for k in range(3):
        p[:, k] = c[k] + s * (p[:, k] - c[k])
    c[3:12] = c[3:12] * s


def _pressure_atm(virial: float, volume: float) -> float:
    return virial / (3 * volume) * KATM if volume > 0 else 0.0   # pressure_atm (field.cpp:2606-2609)


# --- the stage chain -------------------------------------------------------------------------------------------------

def _relax_once(ev, x: np.ndarray, cell: np.ndarray, o: RelaxOptions) -> dict:
    ff = ev.ff
    mass = float(np.cumsum(ff.mass)[-1]) if ff.natoms else 0.0   # summed in atom order, as System::total_mass
    density_of = (lambda c: mass / KNA / (_volume(c) * 1e-24) if _valid(c) else 0.0)
    rep = {"stages": [], "notes": [], "iterations": 0, "evaluations": 0}
    cap_final = o.pushoff_cap if o.pushoff_cap > 0 else (o.pushoff_caps[-1] if o.pushoff_caps else 500.0)
    caps_list = [c for c in o.pushoff_caps if c < cap_final * (1 - 1e-9)] + [cap_final]

    def soft(cap):   # a force cap runs on the FP64 path, as the reference's capped evaluator
        return dataclasses.replace(o.energy, force_cap=float(cap), coulomb=False, precision="double")

    fixed = None if o.fixed is None else list(o.fixed)
    if o.pushoff and o.pushoff_ramp_ps > 0:
        if fixed is not None and any(fixed):
            raise ValueError("push-off dynamics with held atoms: the device dynamics holds no atoms")
        segs = max(1, o.pushoff_ramp_segments)
        c0 = min(caps_list[0], cap_final)
        steps = max(1, int(_round(o.pushoff_ramp_ps * 1000.0 / 1.0 / segs)))
        v = None
        for k in range(segs):
            cap = cap_final if segs == 1 else c0 * (cap_final / c0) ** (k / (segs - 1))
            eo = soft(cap)
            ev.set_options(eo)
            md = DynamicsOptions(dt=1.0, steps=steps, temperature=o.pushoff_temperature, thermostat="bussi", tau_t=100.0, seed=1,
                                 thermo_every=max(1, steps // 40), frame_every=0, new_velocities=k == 0, step_offset=steps * k, energy=eo)
            out = ev.run(x, cell, md, v=v)
            x[:] = out["x"].reshape(x.shape)
            v = out["v"]
            nm = "push-off MD, force cap %.3g" % cap
            rep["stages"].append({"name": nm, "iterations": steps, "energy": out["thermo"][-1]["potential"] if out["thermo"] else 0.0,
                                  "fmax": 0.0, "density": 0.0, "pressure": 0.0, "stopped_by": "time"})
        rep["notes"].append("push-off MD: %g ps NVT at %g K, LJ force cap raised from %g to %g kcal/mol/Å in %d steps"
                            % (o.pushoff_ramp_ps, o.pushoff_temperature, c0, cap_final, segs))

    if _valid(cell):
        a, b, c = cell[3:6], cell[6:9], cell[9:12]
        v = _volume(cell)
        w = min(v / math.sqrt(_dot(_cross(b, c), _cross(b, c))), v / math.sqrt(_dot(_cross(c, a), _cross(c, a))),
                v / math.sqrt(_dot(_cross(a, b), _cross(a, b))))
        if o.target_density > 0 and w * math.cbrt(density_of(cell) / o.target_density) < 2 * o.energy.cutoff:
            rep["notes"].append("the cell will be narrower than twice the cut-off; periodic images are included in the pair list")
    elif o.target_density > 0 or o.relax_box:
        raise FieldError("compression and box relaxation need a periodic cell")

    hold = None
    if fixed is not None:
        hold = np.zeros(x.size, dtype=bool)
        for i, fl in enumerate(fixed[: x.size // 3]):
            for k in range(3):
                if fl == 1 or (int(fl) >> (k + 1)) & 1:
                    hold[3 * i + k] = True

    def free_fmax(f):
        g = np.asarray(f, dtype=np.float64).reshape(-1).copy()
        if hold is not None:
            g[hold] = 0.0
        return max_force(g)

    ev.set_options(o.energy)
    t, f = ev.compute(x, cell)
    rep["initial"], rep["fmax_initial"], rep["density_initial"] = t, free_fmax(f), density_of(cell)

    dens = []
    if o.target_density > 0 and rep["density_initial"] > 0:
        d = rep["density_initial"]
        step = max(0.005, o.compress_step)
        if o.target_density > d:
            while d < o.target_density * (1 - 1e-9):
                d = min(o.target_density, d * (1 + step))
                dens.append(d)
        else:
            while d > o.target_density * (1 + 1e-9):
                d = max(o.target_density, d / (1 + step))
                dens.append(d)

    def minimise_here(mo, name):
        st = minimise(ev, x, cell, mo, name)
        x[:] = st.pop("x").reshape(x.shape)
        rep["evaluations"] += st.pop("evaluations")
        return st

    def run(name, eo, mo):
        ev.set_options(eo)
        rho = density_of(cell)
        st = minimise_here(mo, name)
        st["density"] = rho
        tt, _ = ev.compute(x, cell)
        rep["evaluations"] += 1
        st["pressure"] = _pressure_atm(tt["virial"], _volume(cell)) if _valid(cell) else 0.0
        rep["iterations"] += st["iterations"]
        rep["stages"].append(st)
        return st

    quick = dataclasses.replace(o, method="fire", ftol=max(o.ftol, 5.0), max_iterations=min(o.max_iterations, 400))
    if o.pushoff:
        for cap in caps_list:
            run("push-off, force cap %g" % cap, soft(cap), quick)

    loose = dataclasses.replace(o, ftol=max(o.ftol, 2.0), max_iterations=min(o.max_iterations, 1500))
    for d in dens:
        _scale_affine(x, cell, math.cbrt(density_of(cell) / d))
        nm = "compress to %.3f g/cm³" % d
        ev.set_options(soft(100))
        minimise_here(quick, nm)
        run(nm, o.energy, loose)

    last = run("minimise", o.energy, o)

    if o.relax_box and o.box_anisotropic:
        if sum(abs(float(q)) for q in (cell[4], cell[5], cell[6], cell[8], cell[9], cell[10])) > 1e-6:
            raise FieldError("relaxing the box axis by axis needs an orthorhombic cell (right angles, axes along x, y and z)")
        bulk, lnl_prev, p_prev, max_step = [3.0e4] * 3, [0.0] * 3, [0.0] * 3, [0.02] * 3
        have_prev, cycles, st = False, 0, dict(last)

        def diag():
            tt, _ = ev.compute(x, cell)
            rep["evaluations"] += 1
            out = [tt["w"][k] / _volume(cell) * KATM for k in range(3)]
            st["pressure"] = (out[0] + out[1] + out[2]) / 3
            return out

        pk = diag()
        while cycles < o.box_cycles:
            if all(not o.box_axes[k] or abs(pk[k] - o.pressure) < o.pressure_tol for k in range(3)):
                break
            p = x.reshape(-1, 3)
            for k in range(3):
                if not o.box_axes[k]:
                    continue
                lnl = math.log(abs(float(cell[3 + 4 * k])))
                if have_prev and abs(lnl - lnl_prev[k]) > 1e-9:
                    b = -(pk[k] - p_prev[k]) / (lnl - lnl_prev[k])
                    if 1e3 < b < 5e6:
                        bulk[k] = b
                    if (pk[k] - o.pressure) * (p_prev[k] - o.pressure) < 0:
                        max_step[k] *= 0.5
                lnl_prev[k], p_prev[k] = lnl, pk[k]
                dl = min(max((pk[k] - o.pressure) / bulk[k], -max_step[k]), max_step[k])
                mu = math.exp(dl)
                p[:, k] = cell[k] + mu * (p[:, k] - cell[k])
                for e in (3, 6, 9):
                    cell[e + k] *= mu
            have_prev = True
            ev.set_options(o.energy)
            rho = density_of(cell)
            st = minimise_here(o, "box")
            rep["iterations"] += st["iterations"]
            st["density"] = rho
            pk = diag()
            cycles += 1
        st["name"] = "box relaxed axis by axis to Pxx %.0f · Pyy %.0f · Pzz %.0f atm in %d cycles%s" % (
            pk[0], pk[1], pk[2], cycles, "" if all(o.box_axes) else " (only the chosen axes moved)")
        rep["stages"].append(st)
        if any(o.box_axes[k] and abs(pk[k] - o.pressure) >= o.pressure_tol for k in range(3)):
            rep["notes"].append("the box's axis pressures did not all reach the tolerance in %d cycles" % o.box_cycles)
        rep["notes"].append("box relaxation is 0 K mechanical equilibrium; the density at a temperature needs Dynamics (NPT)")
        last = st
    elif o.relax_box:
        bulk, lnv_prev, p_prev, have_prev, max_step, cycles = 3.0e4, 0.0, 0.0, False, 0.03, 0
        st = dict(last)
        while cycles < o.box_cycles:
            p = st["pressure"]
            if abs(p - o.pressure) < o.pressure_tol:
                break
            lnv = math.log(_volume(cell))
            if have_prev and abs(lnv - lnv_prev) > 1e-9:
                b = -(p - p_prev) / (lnv - lnv_prev)
                if 1e3 < b < 5e6:
                    bulk = b
                if (p - o.pressure) * (p_prev - o.pressure) < 0:
                    max_step *= 0.5
            lnv_prev, p_prev, have_prev = lnv, p, True
            dlnv = min(max((p - o.pressure) / bulk, -max_step), max_step)
            _scale_affine(x, cell, math.exp(dlnv / 3))
            ev.set_options(o.energy)
            rho = density_of(cell)
            st = minimise_here(o, "box")
            tt, _ = ev.compute(x, cell)
            rep["evaluations"] += 1
            st["pressure"] = _pressure_atm(tt["virial"], _volume(cell))
            st["density"] = rho
            rep["iterations"] += st["iterations"]
            cycles += 1
        st["name"] = "box relaxed to %.0f atm in %d cycles" % (st["pressure"], cycles)
        rep["stages"].append(st)
        if abs(st["pressure"] - o.pressure) >= o.pressure_tol:
            rep["notes"].append("box pressure did not reach the tolerance in %d cycles" % o.box_cycles)
        rep["notes"].append("box relaxation is 0 K mechanical equilibrium; the density at a temperature needs Dynamics (NPT)")
        last = st

    t, f = ev.compute(x, cell)
    rep["final"], rep["fmax_final"], rep["density_final"] = t, free_fmax(f), density_of(cell)
    rep["pressure_final"] = _pressure_atm(t["virial"], _volume(cell)) if _valid(cell) else 0.0
    rep["list_builds"] = ev.list_builds()
    rep["converged"] = last["stopped_by"] in ("force", "energy")
    if not rep["converged"]:
        rep["notes"].append("the final minimisation stopped by %s before the force tolerance" % last["stopped_by"])
    return rep


def relax(ev, x, cell, opts: RelaxOptions | None = None) -> dict:
    """relax (relax.cpp:343-369) on the evaluator's engine: the stage chain, then up to three rounds of linear-angle kicks
    and a plain minimisation. Returns the report ({stages, initial, final, fmax_initial, fmax_final, density_initial,
    density_final, pressure_final, iterations, evaluations, converged, notes}) with the relaxed x (N x 3) and cell."""
    o = opts or RelaxOptions()
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1)).copy()
    cell = cell_array(cell).copy()
    rep = _relax_once(ev, x, cell, o)
    for rnd in (1, 2, 3):
        k = kick_linear_angles(x, cell, ev.ff, 7919 * rnd + ev.ff.natoms, 172.0, o.fixed)
        if k == 0:
            break
        again = dataclasses.replace(o, pushoff=False, target_density=0.0, relax_box=False)
        r2 = _relax_once(ev, x, cell, again)
        for key in ("final", "fmax_final", "converged"):
            rep[key] = r2[key]
        rep["iterations"] += r2["iterations"]
        rep["evaluations"] += r2["evaluations"]
        rep["notes"].append("%d %s stuck at 180° on a bent centre (a saddle: no force there, unstable in dynamics) — the centre "
                            "moved 0.15 Å off the line and minimised again" % (k, "angle" if k == 1 else "angles"))
    ev.set_options(o.energy)
    rep["x"], rep["cell"] = x.reshape(-1, 3), cell
    return rep
