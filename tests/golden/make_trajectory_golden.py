"""Makes tests/golden/trajectory_sha256.json: the SHA-256 of each file the reference's caps::write_trajectory
(core/src/io_traj.cpp:47, built into oracle/_ref by oracle/Makefile) writes for the seeded writer cases of
tests/fixtures.py (every cell shape × .lammpstrj / .dcd / .trr, title "golden", dt 2 fs), so the streaming writers are
checked against the reference's bytes where the reference is not built.

    python tests/golden/make_trajectory_golden.py
"""
from __future__ import annotations

import hashlib
import json
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import ref  # noqa: E402
from tests.fixtures import TRAJ_CELLS, TRAJ_FORMATS, trajectory_case  # noqa: E402


def main():
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for cell in TRAJ_CELLS:
            ids, mols, types, frames = trajectory_case(cell)
            for ext in TRAJ_FORMATS:
                p = Path(d) / f"{cell}.{ext}"
                ref.write_trajectory(p, frames, ids, mols, types, title="golden", dt_fs=2.0)
                out[f"{cell}.{ext}"] = hashlib.sha256(p.read_bytes()).hexdigest()
    (HERE / "trajectory_sha256.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()
