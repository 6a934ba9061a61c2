"""Energy minimisation on a device engine: the reference's minimise (core/src/relax.cpp:65-284), its four methods
(steepest descent, conjugate gradients, L-BFGS, FIRE), held atoms and distance and dihedral restraints, with every
energy and force evaluation on one persistent device engine (the force field uploaded once, the cluster list rebuilt
only when atoms move past the skin). The iteration itself (directions, the backtracking line search, the L-BFGS
history) is host arithmetic on 3N-vectors, as in the reference; only the evaluations are on the device.
"""
from __future__ import annotations

import math
from collections import deque
from dataclasses import dataclass, field

import numpy as np

METHODS = {"sd": "sd", "steepest": "sd", "cg": "cg", "lbfgs": "lbfgs", "l-bfgs": "lbfgs", "fire": "fire"}


@dataclass
class MinimiseOptions:
    """The fields of caps::RelaxOptions (core/include/caps/relax.hpp:27-55) that minimise reads."""
    method: str = "lbfgs"
    ftol: float = 0.5              # stop when the largest atomic force is below this, kcal/mol/Å
    etol: float = 1e-8             # or when the relative energy change per step is below this
    max_iterations: int = 5000
    fixed: list | None = None      # per atom: 1 held in place; bits 1-3 (2, 4, 8) hold only x, y, z
    restraints: list = field(default_factory=list)            # (i, j, r0 Å, k kcal/mol/Å²): k (r - r0)^2
    dihedral_restraints: list = field(default_factory=list)   # (i, j, k, l, phi0 degrees, kphi kcal/mol/rad²): kphi (phi - phi0)^2


def max_force(f: np.ndarray) -> float:
    """The largest atomic force (relax.cpp:47-51)."""
    f = f.reshape(-1, 3)
    return float(math.sqrt(float(np.max(np.einsum("ij,ij->i", f, f))))) if f.size else 0.0


def _minimum_image(cell: np.ndarray, d: np.ndarray) -> np.ndarray:
    h = np.asarray(cell[3:12], dtype=np.float64).reshape(3, 3).T   # columns a, b, c
    s = np.linalg.solve(h, d)
    return h @ (s - np.round(s))


def minimise(ev, x, cell, opts: MinimiseOptions, name: str = "minimise") -> dict:
    """minimise (relax.cpp:65) with the evaluator's device engine. Returns {name, iterations, energy, fmax, stopped_by
    ("force", "energy", "iterations", "line search"), evaluations, x (the minimised positions, N x 3)}."""
    method = METHODS.get(opts.method.lower())
    if method is None:
        raise ValueError(f"unknown minimiser '{opts.method}' (sd, cg, lbfgs, fire)")
    cell = np.asarray(cell, dtype=np.float64).reshape(-1)
    x = np.asarray(x, dtype=np.float64).reshape(-1).copy()
    n3 = x.size
    fixed = None if opts.fixed is None else np.asarray(opts.fixed, dtype=np.int64)
    hold = None
    if fixed is not None and fixed.any():
        hold = np.zeros(n3, dtype=bool)
        for i, fl in enumerate(fixed[: n3 // 3]):
            for k in range(3):
                if fl == 1 or (fl >> (k + 1)) & 1:
                    hold[3 * i + k] = True
    nev = 0

    def evaluate(p: np.ndarray):
        nonlocal nev
        nev += 1
        terms, f = ev.compute(p, cell)
        f = np.asarray(f, dtype=np.float64).reshape(-1).copy()
        en = float(terms["total"])
        for (i, j, r0, k) in opts.restraints:
            dv = _minimum_image(cell, p[3 * j:3 * j + 3] - p[3 * i:3 * i + 3])
            r = float(np.linalg.norm(dv))
            if r < 1e-9:
                continue
            en += k * (r - r0) * (r - r0)
            g = 2 * k * (r - r0) / r
            f[3 * j:3 * j + 3] -= g * dv
            f[3 * i:3 * i + 3] += g * dv
        for (i, j, kk, l, phi0, kphi) in opts.dihedral_restraints:
            at = lambda a: p[3 * a:3 * a + 3]
            b1 = _minimum_image(cell, at(j) - at(i))
            b2 = _minimum_image(cell, at(kk) - at(j))
            b3 = _minimum_image(cell, at(l) - at(kk))
            m, nn = np.cross(b1, b2), np.cross(b2, b3)
            m2, n2, lb2 = float(m @ m), float(nn @ nn), float(np.linalg.norm(b2))
            if m2 < 1e-12 or n2 < 1e-12 or lb2 < 1e-9:
                continue
            phi = math.atan2(lb2 * float(b1 @ nn), float(m @ nn))
            dphi = phi - phi0 * math.pi / 180.0
            dphi -= 2 * math.pi * round_half_away(dphi / (2 * math.pi))
            en += kphi * dphi * dphi
            dE = 2 * kphi * dphi
            gi, gl = m * (-lb2 / m2), nn * (lb2 / n2)
            s1, s3 = float(b1 @ b2) / (lb2 * lb2), float(b3 @ b2) / (lb2 * lb2)
            gj, gk = gi * (-s1 - 1) + gl * s3, gi * s1 + gl * (-s3 - 1)
            f[3 * i:3 * i + 3] -= dE * gi
            f[3 * j:3 * j + 3] -= dE * gj
            f[3 * kk:3 * kk + 3] -= dE * gk
            f[3 * l:3 * l + 3] -= dE * gl
        if hold is not None:
            f[hold] = 0.0
        return en, f

    e, f = evaluate(x)
    fmax = max_force(f)
    it = 0
    stopped = "force" if fmax < opts.ftol else "iterations"
    if method == "fire":
        nmin, finc, fdec, astart, falpha, dtmax, maxstep = 5, 1.1, 0.5, 0.1, 0.99, 0.5, 0.1
        dt, alpha, npos = 0.05, astart, 0
        v = np.zeros(n3)
        while it < opts.max_iterations and stopped != "force":
            pw = float(f @ v)
            if pw > 0:
                vn, fnn = math.sqrt(float(v @ v)), math.sqrt(float(f @ f))
                v = (1 - alpha) * v + alpha * vn * f / max(fnn, 1e-300)
                npos += 1
                if npos > nmin:
                    dt, alpha = min(dt * finc, dtmax), alpha * falpha
            else:
                v[:] = 0.0
                dt *= fdec
                alpha, npos = astart, 0
            v += dt * f
            d = dt * v
            md = max_force(d)
            if md > maxstep:
                d *= maxstep / md
            x += d
            e, f = evaluate(x)
            fmax = max_force(f)
            if fmax < opts.ftol:
                stopped = "force"
            it += 1
    else:
        mhist = 10
        S, Y, rho = deque(), deque(), deque()
        fprev, dprev = None, np.zeros(n3)
        cg_restarted = False
        step = 0.1
        step_max = 0.3 if method == "sd" else 0.5
        while it < opts.max_iterations and stopped != "force":
            if method == "sd":
                d = f.copy()
            elif method == "cg":
                if fprev is None:
                    d = f.copy()
                else:
                    den = float(fprev @ fprev)
                    num = float(f @ (f - fprev))
                    beta = max(0.0, num / den) if den > 0 else 0.0
                    d = f + beta * dprev
            else:   # L-BFGS two-loop on the gradient g = -f
                q = -f.copy()
                al = [0.0] * len(S)
                for jj in range(len(S) - 1, -1, -1):
                    al[jj] = rho[jj] * float(S[jj] @ q)
                    q -= al[jj] * Y[jj]
                gamma = float(S[-1] @ Y[-1]) / float(Y[-1] @ Y[-1]) if S else 1.0 / 300.0
                q *= gamma
                for jj in range(len(S)):
                    b = rho[jj] * float(Y[jj] @ q)
                    q += S[jj] * (al[jj] - b)
                d = -q
            slope = float(f @ d)
            if slope <= 0:
                d = f.copy()
                slope = float(f @ f)
                S.clear(), Y.clear(), rho.clear()
            md = max_force(d)
            a = min(1.0, step_max / md) if (method == "lbfgs" and S) else step / md
            ok, en, xn, fn = False, 0.0, None, None
            for _ in range(30):
                xn = x + a * d
                en, fn = evaluate(xn)
                if en <= e - 1e-4 * a * slope:
                    ok = True
                    break
                a *= 0.5
            if ok and method == "cg":
                curv = en - e + a * slope
                if curv > 0:
                    aq = 0.5 * slope * a * a / curv
                    if 0 < aq < 4 * a and abs(aq - a) > 1e-3 * a and aq * md <= step_max:
                        xq = x + aq * d
                        eq, fq = evaluate(xq)
                        if eq < en:
                            xn, fn, en, a = xq, fq, eq, aq
            if not ok:
                if S or fprev is not None:   # start over from steepest descent once
                    S.clear(), Y.clear(), rho.clear()
                    fprev = None
                    step = 0.02
                    it += 1
                    continue
                stopped = "line search"
                break
            moved = a * md
            step = min(max(moved * 1.5, 1e-4), step_max)
            if method == "lbfgs":
                s_, y_ = xn - x, f - fn
                sy = float(s_ @ y_)
                if sy > 1e-10:
                    S.append(s_), Y.append(y_), rho.append(1.0 / sy)
                    if len(S) > mhist:
                        S.popleft(), Y.popleft(), rho.popleft()
            fprev, dprev = f, d
            de = e - en
            x, f, e = xn, fn, en
            fmax = max_force(f)
            if fmax < opts.ftol:
                stopped = "force"
            elif 0 <= de < opts.etol * max(1.0, abs(e)):
                if method == "cg" and not cg_restarted:
                    cg_restarted = True
                    fprev = None
                    step = 0.1
                    it += 1
                    continue
                stopped = "energy"
                it += 1
                break
            else:
                cg_restarted = False
            it += 1
    return {"name": name, "iterations": it, "energy": e, "fmax": fmax, "stopped_by": stopped, "evaluations": nev, "x": x.reshape(-1, 3)}


def round_half_away(v: float) -> float:
    """std::round rounds halves away from zero."""
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)
