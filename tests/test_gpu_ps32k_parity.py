"""Parity at the benchmark's own cell: the 32,000-atom polystyrene PME melt (40 chains x 50 units x 16 atoms, r_c 12 Å
with a 2 Å skin, PME rtol 1e-5, 1 Å spacing, order 4, tail correction on) against the reference's Evaluator::compute
(oracle/_ref, the reference core built from its sources) on the same frames.

FP64 path: every energy term within 1e-12 relative (plus 1e-9 kcal/mol absolute), the virial tensor within 1e-11 of the
virial, forces within 1e-12 (RMS) and 1e-11 (largest component) relative to the RMS force: the bar of the golden-fixture
tests, here at the size every benchmark number is quoted on. Mixed path: RMS relative force error within 5e-6 of the
reference's FP64 forces (the target precision), per-atom and energy errors within the reference's own mixed
tolerances, and no worse than 1.5x the reference's own mixed kernel on the same frame.

Two frames: the committed start structure, and the end of 100 FP64 steps of Nose-Hoover dynamics with SHAKE from it.
"""
import os

import numpy as np
import pytest

from tests.fixtures import ps32k, ps32k_options, rel_max, rel_rms

pytestmark = pytest.mark.gpu

TERMS = ["bond", "angle", "dihedral", "improper", "vdw", "coulomb"]


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built (make -C oracle)")
    return ref


@pytest.fixture(scope="module")
def frames():
    """[(x, cell, oracle FP64 terms, oracle FP64 forces, oracle mixed forces)] for the two frames."""
    from caps_b200 import DynamicsOptions, Evaluator
    ref = _ref()
    ff, x, v, cell = ps32k()
    o = DynamicsOptions(dt=1.0, steps=100, temperature=500.0, thermostat="nose-hoover", tau_t=100.0, constraints="h-bonds", seed=3,
                        thermo_every=100, energy=ps32k_options("double"))
    ev = Evaluator(ff, o.energy)
    x1 = ev.run(x, cell, o, v=v)["x"]
    ev.close()
    threads = os.cpu_count() or 1
    out = []
    for xx in (x, x1):
        t, f = ref.compute(ff, ps32k_options("double"), xx, cell, threads=threads)
        _, fm = ref.compute(ff, ps32k_options("mixed"), xx, cell, threads=threads)
        out.append((xx, cell, t, f, fm))
    return ff, out


@pytest.mark.parametrize("frame", [0, 1])
def test_fp64_matches_reference_at_32k_atoms(frames, frame):
    from caps_b200 import Evaluator
    ff, fr = frames
    x, cell, ref_t, ref_f, _ = fr[frame]
    ev = Evaluator(ff, ps32k_options("double"))
    t, f = ev.compute(x, cell)
    ev.close()
    for k in TERMS:
        assert abs(t[k] - ref_t[k]) <= 1e-12 * abs(ref_t[k]) + 1e-9, (k, t[k], ref_t[k])
    for c in range(6):
        assert abs(t["w"][c] - ref_t["w"][c]) <= 1e-11 * abs(ref_t["virial"]) + 1e-8, ("w", c, t["w"][c], ref_t["w"][c])
    assert abs(t["tail_energy"] - ref_t["tail_energy"]) <= 1e-12 * abs(ref_t["tail_energy"])
    err = rel_rms(f, ref_f)
    assert err <= 1e-12, err
    assert rel_max(f, ref_f) <= 1e-11


@pytest.mark.parametrize("frame", [0, 1])
def test_mixed_within_target_of_reference_fp64_at_32k_atoms(frames, frame):
    from caps_b200 import Evaluator
    ff, fr = frames
    x, cell, ref_t, ref_f, ref_fm = fr[frame]
    ev = Evaluator(ff, ps32k_options("mixed"))
    t, f = ev.compute(x, cell)
    ev.close()
    err = rel_rms(f, ref_f)
    ref_mixed_err = rel_rms(ref_fm, ref_f)
    assert err <= 5e-6, err
    assert err <= max(1e-6, 1.5 * ref_mixed_err), (err, ref_mixed_err)
    per_atom = np.linalg.norm(f - ref_f, axis=1) / np.maximum(np.linalg.norm(ref_f, axis=1), 1e-12)
    assert float(per_atom.max()) <= 1e-3, float(per_atom.max())
    assert abs(t["vdw"] - ref_t["vdw"]) <= 2e-6 * abs(ref_t["vdw"]) + 1e-4, (t["vdw"], ref_t["vdw"])
    assert abs(t["coulomb"] - ref_t["coulomb"]) <= 2e-6 * abs(ref_t["coulomb"]) + 1e-4, (t["coulomb"], ref_t["coulomb"])
    for k in ["bond", "angle", "dihedral", "improper"]:
        assert abs(t[k] - ref_t[k]) <= 1e-5 * abs(ref_t[k]) + 1e-5, (k, t[k], ref_t[k])
    for c in range(6):
        assert abs(t["w"][c] - ref_t["w"][c]) <= 2e-5 * abs(ref_t["virial"]) + 1e-3, ("w", c)
