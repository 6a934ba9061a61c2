"""ORACLE / TEST INFRASTRUCTURE — the reference CAPS core (oracle/_ref/libcaps_ref.so, built by oracle/Makefile from
the reference's own sources plus the C++ restatement of its Fortran PME) driven from Python.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm use this module, as the checker. It takes the same
caps_b200.ForceField the device engine takes and hands it to the reference through oracle/ref_shim.cpp.
"""
from __future__ import annotations

import ctypes as C
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from caps_b200 import _abi  # noqa: E402
from caps_b200.engine import DynamicsOptions, EnergyOptions, cell_array  # noqa: E402
from caps_b200.forcefield import ForceField, read_capsff  # noqa: E402

LIB = Path(__file__).resolve().parent / "_ref" / "libcaps_ref.so"


class TgFit(C.Structure):
    """ref_tg_fit: the reference's glass-transition fit (BilinearFit, core/include/caps/mechanics.hpp:303-311)."""
    _fields_ = [("ok", C.c_int32), ("tg", C.c_double), ("tg_err", C.c_double), ("slope_low", C.c_double), ("slope_high", C.c_double),
                ("value_at_tg", C.c_double), ("alpha_low", C.c_double), ("alpha_high", C.c_double), ("rss", C.c_double),
                ("note", C.c_char * 256)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "note"}
        d["ok"] = bool(d["ok"])
        d["note"] = self.note.decode()
        return d
_lib = None


def available() -> bool:
    return LIB.exists()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise RuntimeError(f"{LIB} is missing: build it with `make -C oracle` where the reference sources are")
        L = C.CDLL(str(LIB))
        L.ref_error.restype = C.c_char_p
        L.ref_compute.argtypes = [C.POINTER(_abi.FF), C.POINTER(_abi.Opts), C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(_abi.Terms), C.c_int]
        L.ref_time_compute.argtypes = [C.POINTER(_abi.FF), C.POINTER(_abi.Opts), C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)]
        L.ref_run.argtypes = [C.POINTER(_abi.FF), C.POINTER(_abi.Opts), C.POINTER(_abi.State), C.POINTER(_abi.MdOpts), C.c_void_p, C.c_int,
                              C.POINTER(_abi.Thermo), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double),
                              _abi.FRAME_FN, C.c_void_p]
        L.ref_request_stop.argtypes = [C.c_int]
        L.ref_ev_create.restype = C.c_void_p
        L.ref_ev_create.argtypes = [C.POINTER(_abi.FF), C.POINTER(_abi.Opts), C.c_int]
        L.ref_ev_set_options.argtypes = [C.c_void_p, C.POINTER(_abi.Opts), C.c_int]
        L.ref_ev_compute.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(_abi.Terms)]
        L.ref_ev_list_builds.argtypes = [C.c_void_p]
        L.ref_ev_destroy.argtypes = [C.c_void_p]
        L.ref_relax.argtypes = [C.POINTER(_abi.FF), C.POINTER(_abi.Opts), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_int, C.c_void_p, C.c_char_p, C.c_int, C.c_char_p, C.c_int]
        L.ref_freeze_compute.argtypes = [C.POINTER(_abi.FF), C.POINTER(_abi.Opts), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.POINTER(_abi.Terms), C.POINTER(C.c_int64), C.c_int]
        L.ref_pairs.argtypes = [C.POINTER(_abi.FF), C.POINTER(_abi.Opts), C.c_void_p, C.c_void_p, C.POINTER(C.c_int64), C.c_int]
        L.ref_reload_compute.argtypes = [C.POINTER(_abi.FF), C.POINTER(_abi.FF), C.POINTER(_abi.Opts), C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.POINTER(_abi.Terms), C.c_int]
        L.ref_write_trajectory.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_int, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_double]
        L.ref_ewald_beta.restype = C.c_double
        L.ref_ewald_beta.argtypes = [C.c_double, C.c_double]
        L.ref_pme_grid.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_void_p]
        L.ref_pme.restype = C.c_double
        L.ref_pme.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int]
        L.ref_ewald.restype = C.c_double
        L.ref_ewald.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
        L.ref_build_ps_gaff.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint64, C.c_char_p]
        L.ref_build_kg.argtypes = [C.c_int, C.c_int, C.c_double, C.c_uint64, C.c_char_p]
        L.ref_fit_tg.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(TgFit)]
        L.ref_run_cooling.argtypes = [C.POINTER(_abi.FF), C.POINTER(_abi.Opts), C.POINTER(_abi.State), C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(TgFit)]
        L.ref_equilibrate.argtypes = [C.POINTER(_abi.FF), C.POINTER(_abi.Opts), C.POINTER(_abi.State), C.POINTER(_abi.MdOpts), C.c_int,
                                      C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.c_void_p]
        L.ref_minimise.argtypes = [C.POINTER(_abi.FF), C.POINTER(_abi.Opts), C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int,
                                   C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]
        _lib = L
    return _lib


def _vp(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def compute(ff: ForceField, opts: EnergyOptions, x, cell, threads: int = 1) -> tuple[dict, np.ndarray]:
    """caps::Evaluator(ff, opts).compute(x, cell) in the reference core."""
    s, keep = ff.to_struct()
    o = opts.to_struct()
    xx = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    c = cell_array(cell)
    f = np.zeros_like(xx)
    t = _abi.Terms()
    if lib().ref_compute(C.byref(s), C.byref(o), _vp(xx), _vp(c), _vp(f), C.byref(t), threads) != 0:
        raise RuntimeError(lib().ref_error().decode())
    return t.as_dict(), f.reshape(-1, 3)


def time_compute(ff: ForceField, opts: EnergyOptions, x, cell, reps: int, threads: int) -> float:
    s, keep = ff.to_struct()
    o = opts.to_struct()
    xx = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    c = cell_array(cell)
    sec = C.c_double()
    if lib().ref_time_compute(C.byref(s), C.byref(o), _vp(xx), _vp(c), reps, threads, C.byref(sec)) != 0:
        raise RuntimeError(lib().ref_error().decode())
    return sec.value


def run(ff: ForceField, x, cell, opts: DynamicsOptions, v=None, threads: int = 1, max_rows: int = 100000, frames: bool = False,
        checkpoints: bool = False, events: list | None = None) -> dict:
    """caps::run_dynamics in the reference core; returns {x, v, cell, thermo, seconds, ns_per_day}, plus "frames" [(x,
    cell, step)] and "checkpoints" [(x, v, cell, step)] when asked for, and "interrupted" (the DynamicsInterrupted text)
    when a stop ended the run. events, when given, receives ("row" | "frame" | "checkpoint", step) in call order."""
    s, keep = ff.to_struct()
    o = opts.energy.to_struct()
    xx = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1)).copy()
    vv = np.zeros_like(xx) if v is None else np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1)).copy()
    c = cell_array(cell).copy()
    st = _abi.State(_vp(xx), _vp(vv), _vp(c), 0 if v is None else 1)
    m = opts.to_struct(ff, keep)
    el = np.ascontiguousarray(ff.element if ff.element is not None else np.full(ff.natoms, 6), dtype=np.int32)
    rows = (_abi.Thermo * max_rows)()
    nrows, sec, nsd = C.c_int(), C.c_double(), C.c_double()
    n = ff.natoms
    fr, ck = [], []

    def _frame(xp, cp, step, user):
        fr.append((np.ctypeslib.as_array(xp, shape=(3 * n,)).copy().reshape(-1, 3), np.ctypeslib.as_array(cp, shape=(12,)).copy(), int(step)))
        if events is not None:
            events.append(("frame", int(step)))

    def _ckpt(xp, vp, cp, step, user):
        ck.append((np.ctypeslib.as_array(xp, shape=(3 * n,)).copy().reshape(-1, 3), np.ctypeslib.as_array(vp, shape=(3 * n,)).copy().reshape(-1, 3),
                   np.ctypeslib.as_array(cp, shape=(12,)).copy(), int(step)))
        if events is not None:
            events.append(("checkpoint", int(step)))

    ff_ = _abi.FRAME_FN(_frame) if frames else _abi.FRAME_FN()
    cf = _abi.CHECKPOINT_FN(_ckpt)
    if checkpoints:
        m.checkpoint = C.cast(cf, C.c_void_p)
    rc = lib().ref_run(C.byref(s), C.byref(o), C.byref(st), C.byref(m), _vp(el), threads, rows, max_rows, C.byref(nrows), C.byref(sec),
                       C.byref(nsd), ff_, None)
    if rc < 0:
        raise RuntimeError(lib().ref_error().decode())
    th = [rows[k].as_dict() for k in range(min(nrows.value, max_rows))]
    if events is not None:
        # the rows arrive through a table, not a callback: put them back in call order, each before its step's frame
        merged, k = [], 0
        for kind, step in events:
            while k < len(th) and th[k]["step"] <= step:
                merged.append(("row", th[k]["step"]))
                k += 1
            merged.append((kind, step))
        merged += [("row", r["step"]) for r in th[k:]]
        events[:] = merged
    out = {"x": xx.reshape(-1, 3), "v": vv.reshape(-1, 3), "cell": c, "thermo": th, "seconds": sec.value, "ns_per_day": nsd.value,
           "frames": fr, "checkpoints": ck}
    if rc == 1:
        out["interrupted"] = lib().ref_error().decode()
    return out


def freeze_compute(ff: ForceField, opts: EnergyOptions, x0, cell0, x1, cell1, threads: int = 1) -> tuple[dict, np.ndarray, int]:
    """Evaluator::freeze_pairs(x0, cell0), then compute(x1, cell1): (terms, forces, pairs())."""
    s, keep = ff.to_struct()
    o = opts.to_struct()
    a = np.ascontiguousarray(np.asarray(x0, dtype=np.float64).reshape(-1))
    b = np.ascontiguousarray(np.asarray(x1, dtype=np.float64).reshape(-1))
    c0, c1 = cell_array(cell0), cell_array(cell1)
    f = np.zeros_like(b)
    t = _abi.Terms()
    npairs = C.c_int64()
    if lib().ref_freeze_compute(C.byref(s), C.byref(o), _vp(a), _vp(c0), _vp(b), _vp(c1), _vp(f), C.byref(t), C.byref(npairs), threads) != 0:
        raise RuntimeError(lib().ref_error().decode())
    return t.as_dict(), f.reshape(-1, 3), npairs.value


def pairs(ff: ForceField, opts: EnergyOptions, x, cell, threads: int = 1) -> int:
    """Evaluator::pairs() after one compute at (x, cell)."""
    s, keep = ff.to_struct()
    o = opts.to_struct()
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    c = cell_array(cell)
    npairs = C.c_int64()
    if lib().ref_pairs(C.byref(s), C.byref(o), _vp(a), _vp(c), C.byref(npairs), threads) != 0:
        raise RuntimeError(lib().ref_error().decode())
    return npairs.value


def reload_compute(ff1: ForceField, ff2: ForceField, opts: EnergyOptions, x, cell, threads: int = 1) -> tuple[dict, np.ndarray]:
    """An evaluator on ff1 computes at (x, cell); its force field becomes ff2 in place and is reloaded; the second
    compute's (terms, forces)."""
    s1, k1 = ff1.to_struct()
    s2, k2 = ff2.to_struct()
    o = opts.to_struct()
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    c = cell_array(cell)
    f = np.zeros_like(a)
    t = _abi.Terms()
    if lib().ref_reload_compute(C.byref(s1), C.byref(s2), C.byref(o), _vp(a), _vp(c), _vp(f), C.byref(t), threads) != 0:
        raise RuntimeError(lib().ref_error().decode())
    return t.as_dict(), f.reshape(-1, 3)


def request_stop(on: bool = True):
    """caps::request_stop in the reference core (its own flag, apart from the device engine's)."""
    lib().ref_request_stop(int(bool(on)))


def write_trajectory(path, frames, ids, mols, types, title: str = "", dt_fs: float = 1.0):
    """caps::write_trajectory on the frames [(x, cell, step)] of atoms with the given ids, mols and types."""
    n = len(ids)
    x = np.ascontiguousarray(np.array([np.asarray(f[0], dtype=np.float64).reshape(-1) for f in frames]).reshape(-1)) if frames else np.zeros(0)
    c = np.ascontiguousarray(np.array([cell_array(f[1]) for f in frames]).reshape(-1)) if frames else np.zeros(0)
    st = np.ascontiguousarray(np.array([int(f[2]) for f in frames], dtype=np.int64))
    ia = np.ascontiguousarray(np.asarray(ids, dtype=np.int64))
    ma = np.ascontiguousarray(np.asarray(mols, dtype=np.int64))
    ta = np.ascontiguousarray(np.asarray(types, dtype=np.int32))
    if lib().ref_write_trajectory(str(path).encode(), n, _vp(ia), _vp(ma), _vp(ta), title.encode(), len(frames), _vp(x), _vp(c), _vp(st),
                                  float(dt_fs)) != 0:
        raise RuntimeError(lib().ref_error().decode())


def fit_tg(T, y, method: int = 0, glassy_max: float = 0.0, rubbery_min: float = 0.0) -> dict:
    """caps::fit_bilinear (method 0) or caps::fit_two_ranges (method 1) on the given points."""
    t = np.ascontiguousarray(np.asarray(T, dtype=np.float64).reshape(-1))
    v = np.ascontiguousarray(np.asarray(y, dtype=np.float64).reshape(-1))
    out = TgFit()
    if lib().ref_fit_tg(_vp(t), _vp(v), int(t.size), int(method), float(glassy_max), float(rubbery_min), C.byref(out)) != 0:
        raise RuntimeError(lib().ref_error().decode())
    return out.as_dict()


def run_cooling(ff: ForceField, x, cell, co, v=None, threads: int = 1, max_points: int = 1000) -> dict:
    """caps::run_cooling in the reference core on one structure; co: a caps_b200.cooling.CoolingOptions. Returns
    {points, fit, x, v, cell}."""
    s, keep = ff.to_struct()
    o = co.energy.to_struct()
    xx = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1)).copy()
    vv = np.zeros_like(xx) if v is None else np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1)).copy()
    c = cell_array(cell).copy()
    st = _abi.State(_vp(xx), _vp(vv), _vp(c), 0 if v is None else 1)
    opt = np.array([co.t_start, co.t_end, co.t_step, co.ps_per_step, co.equilibrate_ps, co.average_from, co.dt, co.tau_t, co.tau_p,
                    co.pressure, co.compressibility, co.glassy_max, co.rubbery_min], dtype=np.float64)
    iopt = np.array([0 if co.barostat.lower() == "none" else 1, co.seed, int(bool(co.new_velocities)), co.property, co.fit], dtype=np.int64)
    el = np.ascontiguousarray(ff.element if ff.element is not None else np.full(ff.natoms, 6), dtype=np.int32)
    pts = np.zeros((max_points, 5))
    npts = C.c_int()
    fit = TgFit()
    if lib().ref_run_cooling(C.byref(s), C.byref(o), C.byref(st), _vp(opt), _vp(iopt), _vp(el), threads, _vp(pts), max_points, C.byref(npts),
                             C.byref(fit)) != 0:
        raise RuntimeError(lib().ref_error().decode())
    keys = ("temperature", "density", "density_err", "specific_volume", "potential")
    points = [dict(zip(keys, map(float, pts[k]))) for k in range(min(npts.value, max_points))]
    return {"points": points, "fit": fit.as_dict(), "x": xx.reshape(-1, 3), "v": vv.reshape(-1, 3), "cell": c}


def equilibrate(ff: ForceField, x, cell, eq, v=None, threads: int = 1) -> dict:
    """caps::equilibrate in the reference core; eq: a caps_b200.equilibrate.EquilibrateOptions. Returns {stages (ps,
    temperature, pressure, density, potential, density_end per stage), x, v, cell}."""
    s, keep = ff.to_struct()
    o = eq.md.energy.to_struct()
    xx = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1)).copy()
    vv = np.zeros_like(xx) if v is None else np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1)).copy()
    c = cell_array(cell).copy()
    st = _abi.State(_vp(xx), _vp(vv), _vp(c), 0 if v is None else 1)
    m = eq.md.to_struct(ff, keep)
    ens = np.array([{"nvt": 0, "npt": 1, "nve": 2}[g.ensemble] for g in eq.stages], dtype=np.int32)
    sd = np.array([[g.ps, g.t_start, g.t_end, g.pressure, g.force_cap] for g in eq.stages], dtype=np.float64).reshape(-1)
    el = np.ascontiguousarray(ff.element if ff.element is not None else np.full(ff.natoms, 6), dtype=np.int32)
    out = np.zeros((len(eq.stages), 6))
    if lib().ref_equilibrate(C.byref(s), C.byref(o), C.byref(st), C.byref(m), len(eq.stages), _vp(ens), _vp(sd), float(eq.thermo_ps), _vp(el),
                             threads, _vp(out)) != 0:
        raise RuntimeError(lib().ref_error().decode())
    keys = ("ps", "temperature", "pressure", "density", "potential", "density_end")
    return {"stages": [dict(zip(keys, map(float, r))) for r in out], "x": xx.reshape(-1, 3), "v": vv.reshape(-1, 3), "cell": c}


def minimise(ff: ForceField, energy: EnergyOptions, x, cell, mo) -> dict:
    """caps::minimise in the reference core; mo: a caps_b200.minimise.MinimiseOptions."""
    s, keep = ff.to_struct()
    o = energy.to_struct()
    xx = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1)).copy()
    c = cell_array(cell).copy()
    code = {"sd": 0, "steepest": 0, "cg": 1, "lbfgs": 2, "l-bfgs": 2, "fire": 3}[mo.method.lower()]
    fixed = None if mo.fixed is None else np.ascontiguousarray(np.asarray(mo.fixed, dtype=np.int8))
    rs = np.ascontiguousarray(np.asarray(mo.restraints, dtype=np.float64).reshape(-1, 4)) if mo.restraints else np.zeros((0, 4))
    ds = np.ascontiguousarray(np.asarray(mo.dihedral_restraints, dtype=np.float64).reshape(-1, 6)) if mo.dihedral_restraints else np.zeros((0, 6))
    res = np.zeros(4)
    stopped = C.c_int()
    if lib().ref_minimise(C.byref(s), C.byref(o), _vp(xx), _vp(c), code, mo.ftol, mo.etol, mo.max_iterations,
                          None if fixed is None else _vp(fixed), len(rs), _vp(rs), len(ds), _vp(ds), _vp(res), C.byref(stopped)) != 0:
        raise RuntimeError(lib().ref_error().decode())
    return {"iterations": int(res[0]), "energy": float(res[1]), "fmax": float(res[2]), "evaluations": int(res[3]),
            "stopped_by": ("force", "energy", "iterations", "line search")[stopped.value], "x": xx.reshape(-1, 3)}


def ewald_beta(rc: float, rtol: float) -> float:
    return lib().ref_ewald_beta(rc, rtol)


def pme_grid(cell, beta: float, spacing: float, order: int) -> list[int]:
    c = cell_array(cell)
    k = np.zeros(3, np.int32)
    lib().ref_pme_grid(_vp(c), beta, spacing, order, _vp(k))
    return [int(v) for v in k]


def pme(x, q, cell, k, order: int, beta: float, threads: int = 1) -> tuple[float, np.ndarray, np.ndarray]:
    xx = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    qq = np.ascontiguousarray(np.asarray(q, dtype=np.float64))
    c = cell_array(cell)
    kk = np.ascontiguousarray(np.asarray(k, dtype=np.int32))
    f = np.zeros_like(xx)
    vir = np.zeros(6)
    e = lib().ref_pme(len(qq), _vp(xx), _vp(qq), _vp(c), _vp(kk), order, beta, _vp(f), _vp(vir), threads)
    return e, f.reshape(-1, 3), vir


def ewald(x, q, cell, kmax, beta: float) -> tuple[float, np.ndarray, np.ndarray]:
    """The reference's plain Ewald reciprocal sum (ewald_reciprocal, core/include/caps/kspace.hpp:28) over
    |m_d| <= kmax[d]: energy, forces, virial (xx yy zz xy xz yz)."""
    xx = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    qq = np.ascontiguousarray(np.asarray(q, dtype=np.float64))
    c = cell_array(cell)
    km = np.ascontiguousarray(np.asarray(kmax, dtype=np.int32))
    f = np.zeros_like(xx)
    vir = np.zeros(6)
    e = lib().ref_ewald(len(qq), _vp(xx), _vp(qq), _vp(c), _vp(km), beta, _vp(f), _vp(vir))
    return e, f.reshape(-1, 3), vir


def build_ps_gaff(chains: int, dp: int, grow_density: float, target_density: float, seed: int):
    """A grown and relaxed atactic polystyrene cell with GAFF (the reference's grow + relax + assign_gaff)."""
    with tempfile.TemporaryDirectory() as d:
        p = str(Path(d) / "cell.bin")
        if lib().ref_build_ps_gaff(chains, dp, grow_density, target_density, seed, p.encode()) != 0:
            raise RuntimeError(lib().ref_error().decode())
        return read_capsff(p)


def build_kg(chains: int, beads: int, density: float, seed: int):
    with tempfile.TemporaryDirectory() as d:
        p = str(Path(d) / "cell.bin")
        if lib().ref_build_kg(chains, beads, density, seed, p.encode()) != 0:
            raise RuntimeError(lib().ref_error().decode())
        return read_capsff(p)


def relax(ff: ForceField, x, cell, ro) -> dict:
    """caps::relax in the reference core (check_cell_fit off); ro: a caps_b200.relax.RelaxOptions. Returns the report
    fields, the stages and the relaxed x (N x 3) and cell."""
    s, keep = ff.to_struct()
    o = ro.energy.to_struct()
    xx = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1)).copy()
    c = cell_array(cell).copy()
    code = {"sd": 0, "steepest": 0, "cg": 1, "lbfgs": 2, "l-bfgs": 2, "fire": 3}[ro.method.lower()]
    opt = np.array([code, ro.ftol, ro.etol, ro.max_iterations, int(ro.pushoff), ro.pushoff_ramp_ps, ro.pushoff_cap, ro.pushoff_temperature,
                    ro.pushoff_ramp_segments, ro.target_density, ro.compress_step, int(ro.relax_box), ro.pressure, ro.pressure_tol,
                    ro.box_cycles, int(ro.box_anisotropic), *[int(bool(a)) for a in ro.box_axes]], dtype=np.float64)
    caps = np.ascontiguousarray(np.asarray(ro.pushoff_caps, dtype=np.float64))
    fixed = None if ro.fixed is None else np.ascontiguousarray(np.asarray(ro.fixed, dtype=np.int8))
    res = np.zeros(16)
    st = np.zeros(6 * 256)
    names, notes = C.create_string_buffer(65536), C.create_string_buffer(65536)
    if lib().ref_relax(C.byref(s), C.byref(o), _vp(xx), _vp(c), _vp(opt), len(caps), _vp(caps), None if fixed is None else _vp(fixed),
                       _vp(res), 256, _vp(st), names, 65536, notes, 65536) != 0:
        raise RuntimeError(lib().ref_error().decode())
    nst = int(res[10])
    nm = names.value.decode().split("\n")[:nst]
    stopped = ("force", "energy", "iterations", "line search", "time")
    stages = [{"name": nm[k], "iterations": int(st[6 * k]), "energy": st[6 * k + 1], "fmax": st[6 * k + 2], "density": st[6 * k + 3],
               "pressure": st[6 * k + 4], "stopped_by": stopped[int(st[6 * k + 5])]} for k in range(min(nst, 256))]
    return {"fmax_initial": res[0], "fmax_final": res[1], "density_initial": res[2], "density_final": res[3], "pressure_final": res[4],
            "iterations": int(res[5]), "evaluations": int(res[6]), "converged": bool(res[7]), "initial_total": res[8], "final_total": res[9],
            "stages": stages, "notes": [n for n in notes.value.decode().split("\n") if n], "x": xx.reshape(-1, 3), "cell": c}


class Evaluator:
    """A persistent caps::Evaluator of the reference core, in caps_b200.Evaluator's calling convention (compute,
    set_options, list_builds, ff): a driver run on it makes the reference's own sequence of calls on one evaluator."""

    def __init__(self, ff: ForceField, options: EnergyOptions, threads: int = 1):
        self.ff, self.options, self.threads = ff, options, threads
        s, self._keep = ff.to_struct()
        o = options.to_struct()
        self.h = lib().ref_ev_create(C.byref(s), C.byref(o), threads)
        if not self.h:
            raise RuntimeError(lib().ref_error().decode())

    def set_options(self, options: EnergyOptions):
        self.options = options
        o = options.to_struct()
        if lib().ref_ev_set_options(self.h, C.byref(o), self.threads) != 0:
            raise RuntimeError(lib().ref_error().decode())

    def compute(self, x, cell):
        xx = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
        c = cell_array(cell)
        f = np.zeros_like(xx)
        t = _abi.Terms()
        if lib().ref_ev_compute(self.h, _vp(xx), _vp(c), _vp(f), C.byref(t)) != 0:
            raise RuntimeError(lib().ref_error().decode())
        return t.as_dict(), f.reshape(-1, 3)

    def list_builds(self) -> int:
        return int(lib().ref_ev_list_builds(self.h))

    def close(self):
        if self.h:
            lib().ref_ev_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
