"""Trajectory files written frame by frame: caps::write_trajectory (core/src/io_traj.cpp:47) for the LAMMPS text dump
(.lammpstrj / .dump, io_lammps.cpp:585-617), LAMMPS's DCD (.dcd, io_binary.cpp:414-462) and GROMACS's TRR (.trr,
io_traj.cpp:81-107), through the engine library's native writer (caps_gpu_traj_* in include/caps_gpu.h).

The reference writes a Trajectory it holds in memory; a TrajectoryWriter takes each frame as it arrives and writes the
same bytes. Given as the `frame` argument of Evaluator.run, the run hands its frames straight to the native writer (no
Python call per frame), on the host while the device integrates the following steps.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .engine import cell_array


class TrajectoryWriter:
    """A trajectory file open for appending frames; the format is the path's extension.

    ids / mols: LAMMPS atom and molecule ids (default 1..N and 1); types: 1-based atom types (default 1); title: the DCD's
    second title line; dt_fs: the time step, for DCD's time unit and TRR's times (step × dt).
    """

    def __init__(self, path, natoms: int, ids=None, mols=None, types=None, title: str = "", dt_fs: float = 1.0):
        self.lib = _abi.load()
        self.natoms = int(natoms)
        self._keep = []

        def arr(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(np.asarray(a, dtype=dt).reshape(-1))
            if a.size != self.natoms:
                raise ValueError("one value per atom")
            self._keep.append(a)
            return a.ctypes.data_as(C.c_void_p)

        h = self.lib.caps_gpu_traj_open(str(path).encode(), self.natoms, arr(ids, np.int64), arr(mols, np.int64), arr(types, np.int32),
                                        (title or "").encode(), float(dt_fs))
        if not h:
            raise OSError(self.lib.caps_gpu_error(None).decode())
        self.h = h
        self.path = str(path)

    @classmethod
    def for_field(cls, path, ff, mols=None, title: str = "", dt_fs: float = 1.0) -> "TrajectoryWriter":
        """A writer for a force field's atoms: ids 1..N, types the field's (1-based)."""
        types = None if ff.type_index is None else np.asarray(ff.type_index) + 1
        return cls(path, ff.natoms, mols=mols, types=types, title=title, dt_fs=dt_fs)

    def append(self, x, cell, step: int):
        if not self.h:
            raise ValueError("the trajectory is closed")
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
        if x.size != 3 * self.natoms:
            raise ValueError("x: 3 coordinates per atom")
        c = cell_array(cell) if cell is not None else np.zeros(12)
        if self.lib.caps_gpu_traj_append(self.h, x.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p), int(step)) != 0:
            raise OSError(self.lib.caps_gpu_error(None).decode())

    __call__ = append

    @property
    def frames(self) -> int:
        return int(self.lib.caps_gpu_traj_frames(self.h)) if self.h else 0

    def native_frame_fn(self):
        """The C frame callback and its user pointer, for caps_gpu_run: frames go to the file with no Python in between."""
        if not self.h:
            raise ValueError("the trajectory is closed")
        addr = C.cast(self.lib.caps_gpu_traj_frame, C.c_void_p).value
        return _abi.FRAME_FN(addr), C.c_void_p(self.h)

    def close(self):
        if self.h:
            h, self.h = self.h, None
            if self.lib.caps_gpu_traj_close(h) != 0:
                raise OSError(self.lib.caps_gpu_error(None).decode())

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_trajectory(path, frames, natoms: int | None = None, ids=None, mols=None, types=None, title: str = "", dt_fs: float = 1.0):
    """caps::write_trajectory for .lammpstrj / .dump / .dcd / .trr: frames is an iterable of (x, cell, step)."""
    frames = list(frames)
    if natoms is None:
        if not frames:
            raise ValueError("natoms is needed without frames")
        natoms = np.asarray(frames[0][0]).size // 3
    with TrajectoryWriter(path, natoms, ids=ids, mols=mols, types=types, title=title, dt_fs=dt_fs) as w:
        for x, cell, step in frames:
            w.append(x, cell, step)
