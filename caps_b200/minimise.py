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
    return float(math.sqrt(float(np.max(f[:, 0] * f[:, 0] + f[:, 1] * f[:, 1] + f[:, 2] * f[:, 2])))) if f.size else 0.0


def dotv(a: np.ndarray, b: np.ndarray) -> float:
    """The reference's dotv (relax.cpp:55-59): the products summed in order, so that the minimiser's path is the
    reference's to the last bit (a BLAS dot sums in another order)."""
    return float(np.cumsum(a * b)[-1]) if a.size else 0.0


# --- the reference's cell geometry (core/src/system.cpp), restated in its operation order ----------------------------

def dot3(a, b) -> float:
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def cross3(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def cell_volume(c) -> float:
    return abs(dot3(c[3:6], cross3(c[6:9], c[9:12])))


def cell_valid(c) -> bool:
    return cell_volume(c) > 1e-9   # Cell::valid (core/src/system.cpp:14)


def round_half_away(v: float) -> float:
    """std::round rounds halves away from zero."""
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


def minimum_image(c, d):
    """Cell::minimum_image (core/src/system.cpp:27-45), the neighbouring images checked for skewed cells."""
    d = tuple(float(q) for q in d)
    if not cell_valid(c):
        return d
    a, b, cc = tuple(float(q) for q in c[3:6]), tuple(float(q) for q in c[6:9]), tuple(float(q) for q in c[9:12])
    v = dot3(a, cross3(b, cc))
    f = [dot3(d, cross3(b, cc)) / v, dot3(d, cross3(cc, a)) / v, dot3(d, cross3(a, b)) / v]
    f = [q - round_half_away(q) for q in f]
    r = tuple(a[k] * f[0] + b[k] * f[1] + cc[k] * f[2] for k in range(3))
    best, out = dot3(r, r), r
    for i in (-1, 0, 1):
        for j in (-1, 0, 1):
            for k in (-1, 0, 1):
                t = tuple(r[m] + a[m] * i + b[m] * j + cc[m] * k for m in range(3))
                q = dot3(t, t)
                if q < best - 1e-12:
                    best, out = q, t
    return r if best == dot3(r, r) else out


def _minimum_image(cell: np.ndarray, d: np.ndarray) -> np.ndarray:
    return np.array(minimum_image(cell, d))


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
            r = math.sqrt(dot3(dv, dv))
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
            m, nn = np.array(cross3(b1, b2)), np.array(cross3(b2, b3))
            m2, n2, lb2 = dot3(m, m), dot3(nn, nn), math.sqrt(dot3(b2, b2))
            if m2 < 1e-12 or n2 < 1e-12 or lb2 < 1e-9:
                continue
            phi = math.atan2(lb2 * dot3(b1, nn), dot3(m, nn))
            dphi = phi - phi0 * math.pi / 180.0
            dphi -= 2 * math.pi * round_half_away(dphi / (2 * math.pi))
            en += kphi * dphi * dphi
            dE = 2 * kphi * dphi
            gi, gl = m * (-lb2 / m2), nn * (lb2 / n2)
            s1, s3 = dot3(b1, b2) / (lb2 * lb2), dot3(b3, b2) / (lb2 * lb2)
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
            pw = dotv(f, v)
            if pw > 0:
                vn, fnn = math.sqrt(dotv(v, v)), math.sqrt(dotv(f, f))
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
                    den = dotv(fprev, fprev)
                    num = dotv(f, f - fprev)
                    beta = max(0.0, num / den) if den > 0 else 0.0
                    d = f + beta * dprev
            else:   # L-BFGS two-loop on the gradient g = -f
                q = -f.copy()
                al = [0.0] * len(S)
                for jj in range(len(S) - 1, -1, -1):
                    al[jj] = rho[jj] * dotv(S[jj], q)
                    q -= al[jj] * Y[jj]
                gamma = dotv(S[-1], Y[-1]) / dotv(Y[-1], Y[-1]) if S else 1.0 / 300.0
                q *= gamma
                for jj in range(len(S)):
                    b = rho[jj] * dotv(Y[jj], q)
                    q += S[jj] * (al[jj] - b)
                d = -q
            slope = dotv(f, d)
            if slope <= 0:
                d = f.copy()
                slope = dotv(f, f)
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
                sy = dotv(s_, y_)
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
