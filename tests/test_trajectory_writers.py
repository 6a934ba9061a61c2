"""The streaming trajectory writers (caps_gpu_traj_*, host code in the engine library) against the reference's
write_trajectory (core/src/io_traj.cpp:47; write_dcd io_binary.cpp:415, write_lammps_dump io_lammps.cpp:612): the same
frames must give the same file, byte for byte — against oracle/_ref where it is built and against the committed SHA-256
of the reference's files (tests/golden/trajectory_sha256.json) everywhere. Needs no GPU."""
import ctypes as C
import hashlib
import json
import struct

import numpy as np
import pytest

from caps_b200 import TrajectoryWriter, write_trajectory
from tests.fixtures import GOLDEN, TRAJ_CELLS, TRAJ_FORMATS, trajectory_case

CASES = [(c, e) for c in TRAJ_CELLS for e in TRAJ_FORMATS]


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def _mine(path, ids, mols, types, frames, title="golden", dt_fs=2.0):
    with TrajectoryWriter(path, len(ids), ids=ids, mols=mols, types=types, title=title, dt_fs=dt_fs) as w:
        for x, cell, step in frames:
            w.append(x, cell, step)
        assert w.frames == len(frames)
    return path.read_bytes()


@pytest.mark.parametrize("cell,ext", CASES)
def test_writer_matches_golden_digest(tmp_path, cell, ext):
    golden = json.loads((GOLDEN / "trajectory_sha256.json").read_text())
    ids, mols, types, frames = trajectory_case(cell)
    data = _mine(tmp_path / f"t.{ext}", ids, mols, types, frames)
    assert hashlib.sha256(data).hexdigest() == golden[f"{cell}.{ext}"]


@pytest.mark.parametrize("cell,ext", CASES)
def test_writer_matches_reference_bytes(tmp_path, cell, ext):
    ref = _ref()
    ids, mols, types, frames = trajectory_case(cell, natoms=23, nframes=3, seed=5)
    ref.write_trajectory(tmp_path / f"r.{ext}", frames, ids, mols, types, title="a title longer than eighty characters " * 3, dt_fs=0.5)
    a = (tmp_path / f"r.{ext}").read_bytes()
    b = _mine(tmp_path / f"m.{ext}", ids, mols, types, frames, title="a title longer than eighty characters " * 3, dt_fs=0.5)
    assert a == b


@pytest.mark.parametrize("ext", ["dcd", "lammpstrj"])
@pytest.mark.parametrize("nframes", [0, 1, 2])
def test_few_frames_match_reference(tmp_path, ext, nframes):
    """No frames (DCD: the header alone, ic[2] = 1; dump: an empty file) and one frame (no step interval)."""
    ref = _ref()
    ids, mols, types, frames = trajectory_case("rotated", natoms=9, nframes=max(nframes, 1))
    frames = frames[:nframes]
    ref.write_trajectory(tmp_path / f"r.{ext}", frames, ids, mols, types, title="golden", dt_fs=2.0)
    assert (tmp_path / f"r.{ext}").read_bytes() == _mine(tmp_path / f"m.{ext}", ids, mols, types, frames)


def test_trr_without_frames_is_refused_like_the_reference(tmp_path):
    w = TrajectoryWriter(tmp_path / "t.trr", 4)
    with pytest.raises(OSError, match="no frames to write"):
        w.close()
    assert not (tmp_path / "t.trr").exists()


def test_unknown_format_and_unwritable_path(tmp_path):
    with pytest.raises(OSError, match="trajectory format 'xyz'"):
        TrajectoryWriter(tmp_path / "t.xyz", 4)
    with pytest.raises(OSError, match="cannot write"):
        TrajectoryWriter(tmp_path / "missing" / "t.dcd", 4)


def test_dcd_header_fields(tmp_path):
    """The control words completed at close: frames, first step, interval, last - first, the unit-cell flag, the
    AKMA time step; the atom count record; one unit-cell record and three coordinate records per frame."""
    ids, mols, types, frames = trajectory_case("orthogonal", natoms=11, nframes=4)
    data = _mine(tmp_path / "t.dcd", ids, mols, types, frames, dt_fs=2.0)
    ic = struct.unpack("<20i", data[8:88])
    assert data[4:8] == b"CORD"
    assert ic[0] == 4 and ic[1] == 1000 and ic[2] == 250 and ic[3] == 750 and ic[10] == 1 and ic[19] == 24
    assert struct.unpack("<f", data[44:48])[0] == np.float32(2.0 / 48.88821)
    assert struct.unpack("<i", data[268:272])[0] == 11
    per_frame = (4 + 48 + 4) + 3 * (4 + 4 * 11 + 4)
    assert len(data) == 276 + 4 * per_frame
    x0 = np.frombuffer(data[276 + 56 + 4:276 + 56 + 4 + 44], dtype="<f4")
    assert np.array_equal(x0, frames[0][0][:, 0].astype(np.float32))


def test_native_frame_callback_writes_the_same_file(tmp_path):
    """caps_gpu_traj_frame, the C frame callback a run hands its frames to, called as the engine calls it."""
    ids, mols, types, frames = trajectory_case("rotated", natoms=13, nframes=3)
    a = _mine(tmp_path / "a.dcd", ids, mols, types, frames)
    w = TrajectoryWriter(tmp_path / "b.dcd", 13, ids=ids, mols=mols, types=types, title="golden", dt_fs=2.0)
    fn, user = w.native_frame_fn()
    for x, cell, step in frames:
        xx = np.ascontiguousarray(x.reshape(-1))
        cc = np.ascontiguousarray(cell)
        fn(xx.ctypes.data_as(C.POINTER(C.c_double)), cc.ctypes.data_as(C.POINTER(C.c_double)), step, user)
    assert w.frames == 3
    w.close()
    assert (tmp_path / "b.dcd").read_bytes() == a


def test_write_trajectory_helper(tmp_path):
    ids, mols, types, frames = trajectory_case("lammps_form", natoms=6, nframes=2)
    write_trajectory(tmp_path / "h.lammpstrj", frames, ids=ids, mols=mols, types=types)
    text = (tmp_path / "h.lammpstrj").read_text().splitlines()
    assert text[0] == "ITEM: TIMESTEP" and text[1] == "1000" and text[3] == "6"
    assert text[4] == "ITEM: BOX BOUNDS xy xz yz pp pp pp"
    assert text[8] == "ITEM: ATOMS id mol type xu yu zu"
    assert text[9].split()[:3] == ["7", "1", "1"]


def test_large_dump_with_edge_values_matches_reference(tmp_path):
    """A frame large enough for the parallel formatter, with the values where fixed-point formatting is delicate:
    exact ties at the fifth decimal (k / 2^17), signed zeros and tiny negatives that print as -0.00000, and numbers too
    long for the formatter's line (printf's own digits)."""
    ref = _ref()
    n = 20011
    rng = np.random.default_rng(9)
    x = rng.normal(0.0, 30.0, size=(n, 3))
    x.reshape(-1)[: 3 * 4000] = np.arange(-6000, 6000) / 131072.0
    x[4000:4010] = [[-0.0, 0.0, -1e-7], [-4.9999e-6, 5e-6, 2.5e-6], [1e15, -1e15, 123456789.123456], [1e120, -3e150, 7.0],
                    [1.0 / 64, -1.0 / 64, 3.0 / 128], [0.000015, -0.000025, 0.000035], [99999.999995, -99999.999995, 0.5e-5],
                    [1e-300, -1e-300, 5e-324], [2.0 ** 40 + 0.5, -(2.0 ** 40) - 0.5, 0.1], [0.3, 0.7, 0.9]]
    ids = np.arange(1, n + 1)
    mols = np.arange(n) // 7 + 1
    types = np.arange(n) % 4 + 1
    frames = [(x, TRAJ_CELLS["rotated"], 0), (x, TRAJ_CELLS["lammps_form"], 10)]
    ref.write_trajectory(tmp_path / "r.lammpstrj", frames, ids, mols, types)
    assert (tmp_path / "r.lammpstrj").read_bytes() == _mine(tmp_path / "m.lammpstrj", ids, mols, types, frames)
