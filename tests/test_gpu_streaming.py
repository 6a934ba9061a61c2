"""Frames, checkpoints and stops of device runs against the reference's run_dynamics (oracle/_ref).

Frames and checkpoints leave the device asynchronously (a snapshot on the device, a copy to pinned memory on a copy
stream, the callback at a later step), yet the callbacks must see what the reference's see: the same steps, the same
states (FP64 runs to 1e-8 Å and Å/fs over tens of steps), in the same order relative to the thermo rows
(dynamics.cpp:754-770). A stop (request_stop) ends the run at the reference's step with its checkpoints and state.
"""
import numpy as np
import pytest

from caps_b200 import (DynamicsInterrupted, DynamicsOptions, EnergyOptions, Evaluator, TrajectoryWriter, request_stop,
                       run_batch)
from tests.fixtures import load

pytestmark = pytest.mark.gpu


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def _opts(**kw):
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision=kw.pop("precision", "double"))
    base = dict(dt=1.0, steps=40, temperature=300.0, thermostat="bussi", tau_t=100.0, thermo_every=10, frame_every=7,
                checkpoint_every=15, seed=4, energy=eo)
    base.update(kw)
    return DynamicsOptions(**base)


class Recorder:
    def __init__(self, stop_at_row=None):
        self.events, self.frames, self.checkpoints, self.stop_at_row = [], [], [], stop_at_row

    def progress(self, row):
        self.events.append(("row", row["step"]))
        if self.stop_at_row is not None and row["step"] == self.stop_at_row:
            request_stop(True)

    def frame(self, x, cell, step):
        self.events.append(("frame", step))
        self.frames.append((x, cell, step))

    def checkpoint(self, x, v, cell, step):
        self.events.append(("checkpoint", step))
        self.checkpoints.append((x, v, cell, step))


def _same_states(a, b, tol=1e-8):
    assert [s[-1] for s in a] == [s[-1] for s in b]
    for p, q in zip(a, b):
        for u, w in zip(p[:-1], q[:-1]):
            assert np.max(np.abs(np.asarray(u) - np.asarray(w))) < tol


@pytest.mark.parametrize("thermostat,frame_every,checkpoint_every", [("bussi", 7, 15), ("none", 10, 10), ("nose-hoover", 1, 4)])
def test_frames_and_checkpoints_follow_reference(thermostat, frame_every, checkpoint_every):
    ref = _ref()
    fx = load("ps_small")
    o = _opts(thermostat=thermostat, frame_every=frame_every, checkpoint_every=checkpoint_every)
    rec = Recorder()
    out = Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o, progress=rec.progress, frame=rec.frame, checkpoint=rec.checkpoint)
    ev = []
    r = ref.run(fx.ff, fx.x, fx.cell, o, frames=True, checkpoints=True, events=ev)
    assert rec.events == ev
    _same_states(rec.frames, r["frames"])
    _same_states(rec.checkpoints, r["checkpoints"])
    assert np.max(np.abs(out["x"] - r["x"])) < 1e-8


def test_stop_in_a_callback_ends_at_the_reference_step():
    """A stop asked for during step 20's callbacks: the run ends at step 20 after its regular checkpoint and the stop's
    own, with the state of step 20 (the reference: the same, its stop asked for from step 20's frame callback)."""
    ref = _ref()
    fx = load("ps_small")
    o = _opts(frame_every=10, checkpoint_every=10)
    rec = Recorder(stop_at_row=20)
    try:
        with pytest.raises(DynamicsInterrupted, match="stopped at step 20") as ei:
            Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o, progress=rec.progress, frame=rec.frame, checkpoint=rec.checkpoint)
    finally:
        request_stop(False)
    assert ei.value.step == 20
    rf, rc = [], []
    try:
        def frame_cb(x, cell, step):
            rf.append((x, cell, step))
            if step == 20:
                ref.request_stop(True)
        r = _run_ref_with_frame_cb(ref, fx, o, frame_cb, rc)
    finally:
        ref.request_stop(False)
    assert "stopped at step 20" in r["interrupted"]
    assert [c[-1] for c in rec.checkpoints] == [10, 20, 20] == [c[-1] for c in rc]
    _same_states(rec.checkpoints, rc)
    st = ei.value.state
    assert np.max(np.abs(st["x"] - r["x"])) < 1e-8 and np.max(np.abs(st["v"] - r["v"])) < 1e-8


def _run_ref_with_frame_cb(ref, fx, o, frame_cb, ckpts):
    """oracle.ref.run with a Python frame callback that may ask the reference to stop."""
    import ctypes as C

    from caps_b200 import _abi
    from caps_b200.engine import cell_array
    s, keep = fx.ff.to_struct()
    eo = o.energy.to_struct()
    xx = np.ascontiguousarray(np.asarray(fx.x, dtype=np.float64).reshape(-1)).copy()
    vv = np.zeros_like(xx)
    c = cell_array(fx.cell).copy()
    vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    st = _abi.State(vp(xx), vp(vv), vp(c), 0)
    m = o.to_struct(fx.ff, keep)
    n = fx.ff.natoms

    def _frame(xp, cp, step, user):
        frame_cb(np.ctypeslib.as_array(xp, shape=(3 * n,)).copy().reshape(-1, 3), np.ctypeslib.as_array(cp, shape=(12,)).copy(), int(step))

    def _ckpt(xp, vp_, cp, step, user):
        ckpts.append((np.ctypeslib.as_array(xp, shape=(3 * n,)).copy().reshape(-1, 3), np.ctypeslib.as_array(vp_, shape=(3 * n,)).copy().reshape(-1, 3),
                      np.ctypeslib.as_array(cp, shape=(12,)).copy(), int(step)))
    ff_, cf = _abi.FRAME_FN(_frame), _abi.CHECKPOINT_FN(_ckpt)
    m.checkpoint = C.cast(cf, C.c_void_p)
    el = np.ascontiguousarray(fx.ff.element if fx.ff.element is not None else np.full(n, 6), dtype=np.int32)
    rows = (_abi.Thermo * 1000)()
    nrows, sec, nsd = C.c_int(), C.c_double(), C.c_double()
    rc = ref.lib().ref_run(C.byref(s), C.byref(eo), C.byref(st), C.byref(m), vp(el), 1, rows, 1000, C.byref(nrows), C.byref(sec), C.byref(nsd),
                           ff_, None)
    assert rc == 1, ref.lib().ref_error().decode()
    return {"x": xx.reshape(-1, 3), "v": vv.reshape(-1, 3), "interrupted": ref.lib().ref_error().decode()}


def test_stop_asked_before_the_run_ends_it_at_step_one():
    fx = load("ps_small")
    o = _opts(frame_every=0, checkpoint_every=0)
    got = []
    request_stop(True)
    try:
        with pytest.raises(DynamicsInterrupted, match="stopped at step 1 ") as ei:
            Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o, checkpoint=lambda x, v, c, s: got.append(s))
    finally:
        request_stop(False)
    assert got == [1] and ei.value.step == 1
    assert len(ei.value.state["thermo"]) == 1   # the row of step 0 only


def test_batch_frames_and_checkpoints_match_single_runs():
    fx = load("ps_small")
    opts = [_opts(seed=4 + r, frame_every=5 + r, checkpoint_every=12, thermo_every=8) for r in range(2)]
    singles = []
    for o in opts:
        rec = Recorder()
        Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o, frame=rec.frame, checkpoint=rec.checkpoint)
        singles.append(rec)
    evs = [Evaluator(fx.ff, o.energy) for o in opts]
    recs = [Recorder() for _ in opts]
    run_batch(evs, [fx.x] * 2, [fx.cell] * 2, opts, frames=[r.frame for r in recs], checkpoints=[r.checkpoint for r in recs])
    for a, b in zip(recs, singles):
        assert a.events == b.events
        _same_states(a.frames, b.frames, tol=1e-12)
        _same_states(a.checkpoints, b.checkpoints, tol=1e-12)


@pytest.mark.parametrize("ext", ["dcd", "lammpstrj", "trr"])
def test_native_writer_streams_the_run_frames(tmp_path, ext):
    """A TrajectoryWriter given as the frame callback: the run's frames go to the file with no Python per frame; the
    file equals the one written from the same run's frames collected in Python."""
    fx = load("ps_small")
    o = _opts(thermostat="none", frame_every=4, checkpoint_every=0, steps=30)
    types = fx.ff.type_index + 1
    w = TrajectoryWriter(tmp_path / f"a.{ext}", fx.ff.natoms, types=types, dt_fs=o.dt)
    Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o, frame=w)
    assert w.frames == 9
    w.close()
    rec = Recorder()
    Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o, frame=rec.frame)
    with TrajectoryWriter(tmp_path / f"b.{ext}", fx.ff.natoms, types=types, dt_fs=o.dt) as w2:
        for f in rec.frames:
            w2.append(*f)
    assert (tmp_path / f"a.{ext}").read_bytes() == (tmp_path / f"b.{ext}").read_bytes()


def test_batch_native_writers_keep_rows_apart(tmp_path):
    fx = load("ps_small")
    opts = [_opts(seed=7 + r, frame_every=6, checkpoint_every=0, thermo_every=10, steps=24) for r in range(2)]
    evs = [Evaluator(fx.ff, o.energy) for o in opts]
    ws = [TrajectoryWriter(tmp_path / f"r{r}.dcd", fx.ff.natoms) for r in range(2)]
    out = run_batch(evs, [fx.x] * 2, [fx.cell] * 2, opts, frames=ws)
    assert [w.frames for w in ws] == [5, 5]
    for w in ws:
        w.close()
    assert [[row["step"] for row in o["thermo"]] for o in out] == [[0, 10, 20, 24]] * 2



def test_stop_ends_every_replica_of_a_batch():
    """A stop asked for before a batch starts ends every replica at step 1, each with its own stop checkpoint, and the
    error carries every replica's state."""
    fx = load("ps_small")
    opts = [_opts(seed=3 + r, frame_every=0, checkpoint_every=0, thermo_every=5) for r in range(2)]
    evs = [Evaluator(fx.ff, o.energy) for o in opts]
    got = [[], []]
    request_stop(True)
    try:
        with pytest.raises(DynamicsInterrupted, match="stopped at step 1 ") as ei:
            run_batch(evs, [fx.x] * 2, [fx.cell] * 2, opts, checkpoints=[lambda x, v, c, s: got[0].append(s), lambda x, v, c, s: got[1].append(s)])
    finally:
        request_stop(False)
    assert got == [[1], [1]]
    assert ei.value.step == 1 and len(ei.value.state) == 2


def test_batch_writer_beside_a_callable_and_none_gets_its_frames(tmp_path):
    """Frame entries of a batch may mix a native writer with a Python callable and None: the writer still receives
    every frame (through its append), the callable its own, and the replica without one none."""
    fx = load("ps_small")
    opts = [_opts(seed=11 + r, frame_every=6, checkpoint_every=0, thermo_every=12, steps=24) for r in range(3)]
    evs = [Evaluator(fx.ff, o.energy) for o in opts]
    w = TrajectoryWriter(tmp_path / "w.dcd", fx.ff.natoms)
    rec = Recorder()
    run_batch(evs, [fx.x] * 3, [fx.cell] * 3, opts, frames=[w, rec.frame, None])
    assert w.frames == 5
    w.close()
    assert [s for _, _, s in rec.frames] == [0, 6, 12, 18, 24]


class _DiskFull(OSError):
    pass


@pytest.mark.parametrize("where", ["checkpoint", "frame", "progress"])
def test_a_raising_callback_ends_the_run_and_reaches_the_caller(where):
    """An exception in a user's callback ends the run (at the next thermo row at the latest) and reaches the caller,
    as an exception thrown by a callback ends the reference's run_dynamics; the run does not go on to its last step."""
    fx = load("ps_small")
    o = _opts(steps=200, thermo_every=10, frame_every=5, checkpoint_every=5)
    calls = []

    def bad(*a):
        calls.append(a[-1] if where != "progress" else a[0]["step"])
        if len(calls) == 2:
            raise _DiskFull("no space left on device")
        return None

    kw = {"checkpoint": bad if where == "checkpoint" else None, "frame": bad if where == "frame" else None,
          "progress": bad if where == "progress" else None}
    rows = []
    if where != "progress":
        kw["progress"] = lambda r: rows.append(r["step"])
    with pytest.raises(_DiskFull):
        Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o, **kw)
    assert len(calls) == 2
    assert not rows or max(rows) <= 30


def test_a_raising_callback_ends_a_batch():
    fx = load("ps_small")
    opts = [_opts(seed=5 + r, steps=200, frame_every=0, checkpoint_every=5, thermo_every=10) for r in range(2)]
    evs = [Evaluator(fx.ff, o.energy) for o in opts]

    def bad(x, v, c, s):
        raise _DiskFull("no space left on device")
    with pytest.raises(_DiskFull):
        run_batch(evs, [fx.x] * 2, [fx.cell] * 2, opts, checkpoints=[None, bad])
