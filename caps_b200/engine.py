"""The reference's Evaluator / run_dynamics interface over the device engine.

Names and meanings follow caps::EnergyOptions, caps::Evaluator (core/include/caps/field.hpp:274-434) and
caps::DynamicsOptions / run_dynamics (core/include/caps/dynamics.hpp:60-180). Every call goes through the C ABI of
include/caps_gpu.h; errors come back as the reference's exception types (FieldError, ValueError for bad arguments,
DynamicsCancelled).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .forcefield import ForceField


class FieldError(RuntimeError):
    """caps::FieldError (core/include/caps/field.hpp:17)."""


class DynamicsCancelled(RuntimeError):
    """caps::DynamicsCancelled (core/include/caps/dynamics.hpp:168)."""


class DeviceError(RuntimeError):
    """A CUDA call failed, or there is no device (the engine has no CPU fallback)."""


class DynamicsInterrupted(RuntimeError):
    """caps::DynamicsInterrupted (core/include/caps/dynamics.hpp:173-176): a stop was asked for (request_stop) and the run
    ended at `step` (with step_offset) after its checkpoint. `state` holds the run's result at that step (x, v, cell,
    thermo rows), as the reference leaves it in the System."""

    def __init__(self, text: str, state: dict | None = None):
        super().__init__(text)
        words = text.split()
        self.step = int(words[3]) if len(words) > 3 and words[3].lstrip("-").isdigit() else -1
        self.state = state


def request_stop(on: bool = True):
    """caps::request_stop (core/include/caps/live.hpp:29): process-wide; every run checks it at each step."""
    _abi.load().caps_gpu_request_stop(int(bool(on)))


def stop_requested() -> bool:
    return bool(_abi.load().caps_gpu_stop_requested())


class _Callbacks:
    """Keeps the first exception raised by a user's progress, frame or checkpoint callback. ctypes cannot carry an
    exception through the C call that invoked the callback, so each wrapper stores it here; the progress wrapper then
    returns non-zero, which ends the run at its next thermo row (as an exception ends the reference's run_dynamics), and
    the caller re-raises the stored exception once the C call has returned."""

    def __init__(self):
        self.error: BaseException | None = None

    def wrap(self, fn):
        def call(*a):
            if self.error is not None:
                return None
            try:
                return fn(*a)
            except BaseException as e:   # noqa: BLE001 — re-raised after the C call returns
                self.error = e
                return None
        return call

    def reraise(self):
        if self.error is not None:
            e, self.error = self.error, None
            raise e


def _raise(code: int, text: str):
    if code == -3 or code == -4:
        raise FieldError(text)
    if code == -5:
        raise DynamicsCancelled(text)
    if code == -2 or code == -6:
        raise DeviceError(text)
    if code == -7:
        raise DynamicsInterrupted(text)
    raise ValueError(text)


@dataclass
class EnergyOptions:
    """caps::EnergyOptions (field.hpp:274-308), the fields the device path takes. precision "mixed" is
    EnergyOptions::mixed = true; the device's mixed form adds bit-reproducible fixed-point force sums."""
    cutoff: float = 10.0
    skin: float = 2.0
    coulomb: bool = True
    electrostatics: str = "dsf"        # "dsf" | "pme"
    dsf_alpha: float = 0.2
    ewald_rtol: float = 1e-5
    pme_spacing: float = 1.0
    pme_order: int = 5
    tail: bool = True
    precision: str = "mixed"           # "mixed" | "double"
    force_cap: float = 0.0
    parts: int = 3

    def to_struct(self) -> _abi.Opts:
        o = _abi.Opts()
        o.cutoff, o.skin, o.coulomb = self.cutoff, self.skin, int(bool(self.coulomb))
        o.electrostatics = 1 if self.electrostatics.lower() == "pme" else 0
        o.dsf_alpha, o.ewald_rtol, o.pme_spacing, o.pme_order = self.dsf_alpha, self.ewald_rtol, self.pme_spacing, self.pme_order
        o.tail = int(bool(self.tail))
        o.precision = 1 if self.precision == "double" else 0
        o.force_cap, o.parts = self.force_cap, self.parts
        return o


THERMOSTATS = {"none": 0, "nve": 0, "bussi": 1, "csvr": 1, "langevin": 2, "baoab": 2, "nose-hoover": 3, "nhc": 3}
# barostat_from_string (dynamics.cpp:36-42)
BAROSTATS = {"none": 0, "crescale": 1, "c-rescale": 1, "berendsen": 2, "mtk": 3, "mttk": 3, "nose-hoover": 3, "parrinello-rahman-mtk": 3}
# constraint_algorithm_from_string (constraints.hpp:22)
CONSTRAINT_ALGORITHMS = {"shake": 0, "lincs": 1}


@dataclass
class DynamicsOptions:
    """caps::DynamicsOptions (dynamics.hpp:60-154), the fields the device step takes."""
    dt: float = 1.0
    steps: int = 10000
    temperature: float = 300.0
    temperature_end: float = -1.0
    thermostat: str = "bussi"
    tau_t: float = 100.0
    barostat: str = "none"
    pressure: float = 1.0
    tau_p: float = 1000.0
    compressibility: float = 4.5e-5
    barostat_every: int = 10
    constraints: str = "none"          # "none" | "h-bonds"
    new_velocities: bool = False
    seed: int = 1
    thermo_every: int = 100
    frame_every: int = 0
    checkpoint_every: int = 0          # steps between checkpoints (0: none), with a checkpoint callback
    step_offset: int = 0
    respa: int = 1
    respa_split: str = "bonded"        # "bonded": bonded terms inner (the reference's split); "pme": PME outer
    hmr: float = 0.0                   # > 0: hydrogen mass repartitioning to this mass (u)
    anisotropic: bool = False          # Berendsen barostat per Cartesian axis
    couple_axis: tuple = (True, True, True)
    axis_pressure: tuple = (float("nan"), float("nan"), float("nan"))   # atm per axis; NaN: `pressure`
    constraint_algorithm: str = "shake"   # "shake" | "lincs" (positions; RATTLE for the velocities either way)
    energy: EnergyOptions = field(default_factory=EnergyOptions)

    def to_struct(self, ff: ForceField, keep: list) -> _abi.MdOpts:
        m = _abi.MdOpts()
        m.dt, m.steps, m.temperature, m.temperature_end = self.dt, self.steps, self.temperature, self.temperature_end
        m.thermostat = THERMOSTATS[self.thermostat.lower()]
        m.tau_t = self.tau_t
        if self.barostat.lower() not in BAROSTATS:
            raise ValueError(f"unknown barostat '{self.barostat}' (none, crescale, berendsen, mtk)")
        m.barostat = BAROSTATS[self.barostat.lower()]
        m.pressure, m.tau_p, m.compressibility, m.barostat_every = self.pressure, self.tau_p, self.compressibility, self.barostat_every
        m.constraints = 0 if self.constraints in ("none", "", None) else 1
        m.new_velocities = int(bool(self.new_velocities))
        m.seed, m.thermo_every, m.frame_every, m.step_offset, m.respa = self.seed, self.thermo_every, self.frame_every, self.step_offset, self.respa
        m.respa_split = {"bonded": 0, "pme": 1}[self.respa_split]
        m.checkpoint_every = int(self.checkpoint_every)
        alg = (self.constraint_algorithm or "shake").lower()
        if alg not in CONSTRAINT_ALGORITHMS:
            raise ValueError(f"unknown constraint algorithm {self.constraint_algorithm!r} (shake | lincs)")
        m.constraint_algorithm = CONSTRAINT_ALGORITHMS[alg]
        m.hmr = float(self.hmr)
        m.anisotropic = int(bool(self.anisotropic))
        m.couple_axes = sum(1 << k for k in range(3) if self.couple_axis[k])
        if self.anisotropic and m.couple_axes == 0:
            raise ValueError("anisotropic pressure coupling needs at least one coupled axis")
        m.axis_pressure_set = sum(1 << k for k in range(3) if not math.isnan(self.axis_pressure[k]))
        for k in range(3):
            m.axis_pressure[k] = 0.0 if math.isnan(self.axis_pressure[k]) else float(self.axis_pressure[k])
        if ff.element is not None:
            h = np.ascontiguousarray((ff.element == 1).astype(np.int8))
            o = np.ascontiguousarray((ff.element == 8).astype(np.int8))
            keep += [h, o]
            m.is_hydrogen = h.ctypes.data_as(C.c_void_p)
            m.is_oxygen = o.ctypes.data_as(C.c_void_p)
        return m


def cell_array(cell) -> np.ndarray:
    """cell[12] = origin, a, b, c (accepts a 3x3 of edge vectors, a 4x3, or 12 numbers)."""
    c = np.asarray(cell, dtype=np.float64).reshape(-1)
    if c.size == 9:
        c = np.concatenate([np.zeros(3), c])
    if c.size != 12:
        raise ValueError("cell: 12 numbers (origin, a, b, c) or 9 (a, b, c)")
    return np.ascontiguousarray(c)


class Evaluator:
    """caps::Evaluator on the device: Evaluator(ff, options); compute(x, cell) -> (terms, forces)."""

    def __init__(self, ff: ForceField, options: EnergyOptions | None = None):
        self.lib = _abi.load()
        self.ff = ff
        self.options = options or EnergyOptions()
        s, keep = ff.to_struct()
        o = self.options.to_struct()
        h = self.lib.caps_gpu_create(C.byref(s), C.byref(o))
        if not h:
            text = self.lib.caps_gpu_error(None).decode()
            if "no CUDA device" in text:
                raise DeviceError(text)
            raise ValueError(text)
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.caps_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != 0:
            _raise(rc, self.lib.caps_gpu_error(self.h).decode())

    def set_options(self, options: EnergyOptions):
        self.options = options
        o = options.to_struct()
        self._check(self.lib.caps_gpu_set_options(self.h, C.byref(o)))

    def energies(self, on: bool):
        self._check(self.lib.caps_gpu_energies(self.h, int(bool(on))))

    def reload(self, ff: ForceField | None = None):
        """Evaluator::reload (field.hpp:349-352): the force field changed (same atoms); set up again from `ff` (default:
        this evaluator's own ForceField object, changed in place)."""
        if ff is not None:
            if ff.natoms != self.ff.natoms:
                raise ValueError("reload: the force field has another number of atoms")
            self.ff = ff
        s, keep = self.ff.to_struct()
        self._check(self.lib.caps_gpu_reload(self.h, C.byref(s)))

    def freeze_pairs(self, x, cell):
        """Evaluator::freeze_pairs (field.hpp:341-346): later computes take exactly the pairs inside the cut-off at
        (x, cell), on the FP64 path, with no list rebuild (small deformations)."""
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
        c = cell_array(cell)
        self._check(self.lib.caps_gpu_freeze_pairs(self.h, x.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p)))

    def unfreeze(self):
        self._check(self.lib.caps_gpu_unfreeze(self.h))

    def pairs(self) -> int:
        """Evaluator::pairs() (field.hpp:348): the atom pairs of the FP64 pair list."""
        v = int(self.lib.caps_gpu_pairs(self.h))
        if v < 0:
            _raise(-1, self.lib.caps_gpu_error(self.h).decode())
        return v

    def threads(self) -> int:
        return int(self.lib.caps_gpu_threads(self.h))

    def compute(self, x, cell) -> tuple[dict, np.ndarray]:
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
        c = cell_array(cell)
        f = np.zeros_like(x)
        t = _abi.Terms()
        self._check(self.lib.caps_gpu_compute(self.h, x.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p),
                                              f.ctypes.data_as(C.c_void_p), C.byref(t)))
        return t.as_dict(), f.reshape(-1, 3)

    def set_timing(self, flush_bytes: int):
        """Measurement mode for run(): per-step CUDA events, an L2 flush of flush_bytes between steps (< 0: off)."""
        self._check(self.lib.caps_gpu_diag_set_timing(self.h, int(flush_bytes)))

    def tuning(self) -> list[int]:
        """The tuned launch shapes (include/caps_gpu_diag.h): entries per work item, pair-grid cut, PME grid cap, bonded
        cap, PME line blocks x, y, z."""
        v = (C.c_int32 * 7)()
        self._check(self.lib.caps_gpu_diag_get_tuning(self.h, C.cast(v, C.c_void_p)))
        return list(v)

    def pin_tuning(self, v):
        """Pins these launch shapes (the seven values tuning() returns); the engine tunes nothing afterwards."""
        a = (C.c_int32 * 7)(*[int(x) for x in v])
        self._check(self.lib.caps_gpu_diag_set_tuning(self.h, C.cast(a, C.c_void_p)))

    def last_step_ms(self) -> float:
        return float(self.lib.caps_gpu_diag_last_step_ms(self.h))

    def step_kernels(self) -> int:
        """Kernel launches in one plain MD step of the last run (the captured graph's kernel nodes)."""
        return int(self.lib.caps_gpu_diag_step_kernels(self.h))

    def kernels_run(self) -> int:
        """Kernels the last run launched in its step loop (graph kernel nodes replayed, thermo-row kernels)."""
        return int(self.lib.caps_gpu_diag_kernels_run(self.h))

    def list_counts(self) -> tuple[int, int]:
        """List builds and dynamic prunes so far (counted on the device)."""
        v = (C.c_int64 * 2)()
        self._check(self.lib.caps_gpu_diag_list_counts(self.h, v))
        return int(v[0]), int(v[1])

    def pair_timing(self, x, cell, launches: int = 50, flush_bytes: int = 0) -> dict:
        """The pair kernel alone: mean launch time and the pairs it evaluates (include/caps_gpu_diag.h)."""
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
        c = cell_array(cell)
        ms, pin, pl, ne = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        self._check(self.lib.caps_gpu_diag_pair_timing(self.h, x.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p), launches,
                                                       int(flush_bytes), C.byref(ms), C.byref(pin), C.byref(pl), C.byref(ne)))
        return {"avg_ms": ms.value, "pairs_in_cutoff": pin.value, "pairs_listed": pl.value, "entries": ne.value}

    def phase_timing(self, x, cell, launches: int = 50, flush_bytes: int = 0) -> dict:
        """The force evaluation's branches timed alone and together, force-only (include/caps_gpu_diag.h): mean ms of
        the bonded branch, PME, the short-range branch and the whole evaluation."""
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
        c = cell_array(cell)
        ms = np.zeros(4)
        self._check(self.lib.caps_gpu_diag_phase_timing(self.h, x.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p), launches,
                                                        int(flush_bytes), ms.ctypes.data_as(C.c_void_p)))
        return dict(zip(("bonded_ms", "pme_ms", "short_range_ms", "forces_ms"), map(float, ms)))

    def steps_per_second(self) -> float:
        """Throughput of the last run (or batch this evaluator was part of): steps per second of device time."""
        return float(self.lib.caps_gpu_last_steps_per_second(self.h))

    def list_builds(self) -> int:
        return int(self.lib.caps_gpu_list_builds(self.h))

    def run(self, x, cell, opts: DynamicsOptions, v=None, progress=None, frame=None, checkpoint=None) -> dict:
        """run_dynamics on this evaluator's force field: returns {x, v, cell, thermo, report, steps_per_second}.

        progress(row) -> False cancels (DynamicsCancelled). frame(x, cell, step) receives each recorded frame, or frame is
        a TrajectoryWriter, whose native writer then takes the frames with no Python call per frame. checkpoint(x, v,
        cell, step) receives each checkpoint (opts.checkpoint_every). A stop asked for with request_stop ends the run
        with DynamicsInterrupted, whose `state` is this method's result at the stopped step."""
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1)).copy()
        vv = np.zeros_like(x) if v is None else np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1)).copy()
        c = cell_array(cell).copy()
        st = _abi.State(x.ctypes.data_as(C.c_void_p), vv.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p),
                        0 if v is None else 1)
        keep: list = []
        m = opts.to_struct(self.ff, keep)
        rows = []
        cb = _Callbacks()

        def _user_progress(d):
            return progress is not None and progress(d) is False

        user_progress = cb.wrap(_user_progress)

        def _prog(row, user):
            d = row.contents.as_dict()
            rows.append(d)
            stop = user_progress(d)
            return 1 if stop or cb.error is not None else 0

        n = self.ff.natoms
        fuser = None
        if frame is None:
            ff_ = _abi.FRAME_FN()
        elif hasattr(frame, "native_frame_fn"):
            ff_, fuser = frame.native_frame_fn()
        else:
            def _frame(xp, cp, step, user):
                frame(np.ctypeslib.as_array(xp, shape=(3 * n,)).copy().reshape(-1, 3), np.ctypeslib.as_array(cp, shape=(12,)).copy(), int(step))
            ff_ = _abi.FRAME_FN(cb.wrap(_frame))
        if checkpoint is not None:
            def _ckpt(xp, vp, cp, step, user):
                checkpoint(np.ctypeslib.as_array(xp, shape=(3 * n,)).copy().reshape(-1, 3), np.ctypeslib.as_array(vp, shape=(3 * n,)).copy().reshape(-1, 3),
                           np.ctypeslib.as_array(cp, shape=(12,)).copy(), int(step))
            cf = _abi.CHECKPOINT_FN(cb.wrap(_ckpt))
            keep.append(cf)
            m.checkpoint = C.cast(cf, C.c_void_p)
        pf = _abi.PROGRESS_FN(_prog)
        buf = C.create_string_buffer(4096)
        rc = self.lib.caps_gpu_run(self.h, C.byref(st), C.byref(m), pf, ff_, fuser, buf, 4096)
        out = {"x": x.reshape(-1, 3), "v": vv.reshape(-1, 3), "cell": c, "thermo": rows, "report": buf.value.decode(),
               "steps_per_second": float(self.lib.caps_gpu_last_steps_per_second(self.h))}
        cb.reraise()
        try:
            self._check(rc)
        except DynamicsInterrupted as e:
            e.state = out
            raise
        return out


def run_dynamics(ff: ForceField, x, cell, opts: DynamicsOptions, v=None, progress=None, frame=None, checkpoint=None) -> dict:
    """caps::run_dynamics on the device (dynamics.hpp:180)."""
    ev = Evaluator(ff, opts.energy)
    try:
        return ev.run(x, cell, opts, v=v, progress=progress, frame=frame, checkpoint=checkpoint)
    finally:
        ev.close()


def run_batch(evaluators: list, xs: list, cells: list, opts: list, vs: list | None = None, frames: list | None = None,
              checkpoints: list | None = None) -> list[dict]:
    """Independent replicas in lock step (caps_gpu_run_batch): one Evaluator, structure and DynamicsOptions per replica,
    all with the same number of steps. Returns one {x, v, cell, thermo} per replica. frames / checkpoints: per replica a
    callback (x, cell, step) / (x, v, cell, step) or None; a frame entry may be a TrajectoryWriter. A stop asked for
    with request_stop raises DynamicsInterrupted, whose `state` is the list of results."""
    R = len(evaluators)
    if not (len(xs) == len(cells) == len(opts) == R) or R == 0:
        raise ValueError("one structure, cell and options per evaluator")
    keep: list = []
    xa, va, ca, st, ms = [], [], [], [], []
    rows: list[list] = [[] for _ in range(R)]
    for r, ev in enumerate(evaluators):
        x = np.ascontiguousarray(np.asarray(xs[r], dtype=np.float64).reshape(-1)).copy()
        v = np.zeros_like(x) if vs is None or vs[r] is None else np.ascontiguousarray(np.asarray(vs[r], dtype=np.float64).reshape(-1)).copy()
        c = cell_array(cells[r]).copy()
        xa.append(x), va.append(v), ca.append(c)
        st.append(_abi.State(x.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p),
                             0 if vs is None or vs[r] is None else 1))
        ms.append(opts[r].to_struct(ev.ff, keep))

    cb = _Callbacks()

    def _prog(row, user):
        rows[replica_of[user]].append(row.contents.as_dict())
        return 1 if cb.error is not None else 0

    frames = list(frames) if frames is not None else [None] * R
    checkpoints = list(checkpoints) if checkpoints is not None else [None] * R
    if len(frames) != R or len(checkpoints) != R:
        raise ValueError("one frame and one checkpoint entry per replica")
    users = (C.c_void_p * R)(*[C.c_void_p(r) for r in range(R)])
    natoms = [ev.ff.natoms for ev in evaluators]
    if all(f is None for f in frames):
        ff_ = _abi.FRAME_FN()
    elif all(hasattr(f, "native_frame_fn") for f in frames):
        ff_ = frames[0].native_frame_fn()[0]
        for r, f in enumerate(frames):
            users[r] = f.native_frame_fn()[1]
    else:
        # writers mixed with callables or None: every frame comes through Python; a writer takes it by append
        def _frame(xp, cp, step, user):
            r = int(user or 0)
            if frames[r] is not None:
                n = natoms[r]
                xa_ = np.ctypeslib.as_array(xp, shape=(3 * n,)).copy().reshape(-1, 3)
                ca_ = np.ctypeslib.as_array(cp, shape=(12,)).copy()
                if hasattr(frames[r], "native_frame_fn"):
                    frames[r].append(xa_, ca_, int(step))
                else:
                    frames[r](xa_, ca_, int(step))
        ff_ = _abi.FRAME_FN(cb.wrap(_frame))
    replica_of = {users[r]: r for r in range(R)}   # progress and frame callbacks get the same user pointer
    for r, ck in enumerate(checkpoints):
        if ck is None:
            continue

        def _ckpt(xp, vp, cp, step, user, ck=ck, n=natoms[r]):
            ck(np.ctypeslib.as_array(xp, shape=(3 * n,)).copy().reshape(-1, 3), np.ctypeslib.as_array(vp, shape=(3 * n,)).copy().reshape(-1, 3),
               np.ctypeslib.as_array(cp, shape=(12,)).copy(), int(step))
        cf = _abi.CHECKPOINT_FN(cb.wrap(_ckpt))
        keep.append(cf)
        ms[r].checkpoint = C.cast(cf, C.c_void_p)
    pf = _abi.PROGRESS_FN(_prog)
    eng = (C.c_void_p * R)(*[ev.h for ev in evaluators])
    sp = (C.c_void_p * R)(*[C.cast(C.pointer(s_), C.c_void_p) for s_ in st])
    mp = (C.c_void_p * R)(*[C.cast(C.pointer(m_), C.c_void_p) for m_ in ms])
    lib = evaluators[0].lib
    rc = lib.caps_gpu_run_batch(eng, sp, mp, R, pf, ff_, users)
    out = [{"x": xa[r].reshape(-1, 3), "v": va[r].reshape(-1, 3), "cell": ca[r], "thermo": rows[r]} for r in range(R)]
    cb.reraise()
    try:
        evaluators[0]._check(rc)
    except DynamicsInterrupted as e:
        e.state = out
        raise
    return out

