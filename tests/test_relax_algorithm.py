"""The relaxation stage chain (caps_b200.relax: push-off stages under rising force caps, compression, the final
minimisation, box relaxation, the linear-angle kicks) against the reference's relax (core/src/relax.cpp:343), both driven
by the reference's own FP64 forces from one persistent evaluator (both make the same calls on an evaluator with the same
list history): the same stages, iteration counts, stops, energies, densities and pressures, and the same end state. Needs
no GPU (the evaluator here is the reference core)."""
import dataclasses

import numpy as np
import pytest

from caps_b200 import EnergyOptions
from caps_b200.relax import RelaxOptions, kick_linear_angles, minimum_image, relax
from tests.fixtures import load


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def RefEvaluator(ref, ff, opts):
    """One persistent reference evaluator (FP64) taking relax's calls: the reference's relax makes the same calls on its
    own evaluator, so both see the same forces to the last bit."""
    return ref.Evaluator(ff, opts)


def _same_report(mine, theirs, tol=1e-9):
    assert [s["name"] for s in mine["stages"]] == [s["name"] for s in theirs["stages"]]
    for a, b in zip(mine["stages"], theirs["stages"]):
        assert a["stopped_by"] == b["stopped_by"] and a["iterations"] == b["iterations"], (a, b)
        for k in ("energy", "fmax", "density", "pressure"):
            assert abs(a[k] - b[k]) <= tol * max(1.0, abs(b[k])) + 1e-6, (a["name"], k, a[k], b[k])
    assert mine["iterations"] == theirs["iterations"] and mine["evaluations"] == theirs["evaluations"]
    assert mine["converged"] == theirs["converged"]
    for k in ("fmax_initial", "fmax_final", "density_initial", "density_final", "pressure_final"):
        assert abs(mine[k] - theirs[k]) <= tol * max(1.0, abs(theirs[k])) + 1e-6, (k, mine[k], theirs[k])
    assert np.max(np.abs(mine["x"] - theirs["x"])) < 1e-6
    assert np.max(np.abs(mine["cell"] - theirs["cell"])) < 1e-9


def test_stage_chain_matches_reference():
    """Push-off under four caps, compression by 8% in two stages, the final L-BFGS and an isotropic box relaxation."""
    ref = _ref()
    fx = load("ps_small")
    eo = EnergyOptions(cutoff=6.0, skin=1.0, electrostatics="pme", pme_order=5, precision="double")
    c = np.asarray(fx.cell, dtype=np.float64)
    ro = RelaxOptions(method="lbfgs", ftol=0.5, max_iterations=40, energy=eo, target_density=1.08 * 1.0 * _density(fx.ff, c),
                      compress_step=0.05, relax_box=True, pressure=1.0, pressure_tol=50.0, box_cycles=3)
    mine = relax(RefEvaluator(ref, fx.ff, eo), fx.x, fx.cell, ro)
    theirs = ref.relax(fx.ff, fx.x, fx.cell, ro)
    assert [s["name"] for s in theirs["stages"]][:5] == ["push-off, force cap 5", "push-off, force cap 20", "push-off, force cap 100",
                                                         "push-off, force cap 500", theirs["stages"][4]["name"]]
    _same_report(mine, theirs)
    assert mine["notes"] == [n for n in theirs["notes"] if not n.startswith(("energy ", "density "))]


def test_anisotropic_box_matches_reference():
    ref = _ref()
    fx = load("ps_small")
    eo = EnergyOptions(cutoff=6.0, skin=1.0, electrostatics="dsf", precision="double")
    ro = RelaxOptions(method="cg", ftol=1.0, max_iterations=30, energy=eo, pushoff=False, relax_box=True, box_anisotropic=True,
                      box_axes=(False, False, True), pressure=1.0, pressure_tol=20.0, box_cycles=3)
    mine = relax(RefEvaluator(ref, fx.ff, eo), fx.x, fx.cell, ro)
    theirs = ref.relax(fx.ff, fx.x, fx.cell, ro)
    _same_report(mine, theirs)
    assert mine["cell"][3] == fx.cell[3] and mine["cell"][11] != fx.cell[11]


def test_linear_angle_kick_matches_reference():
    """A CH centre put on the line of its two partners: relax kicks it 0.15 Å off the line along the reference's random
    direction (max_iterations 0, so nothing else moves)."""
    ref = _ref()
    fx = load("ps_small")
    x = np.array(fx.x, dtype=np.float64)
    i, j, k = (int(v) for v in fx.ff.angle_ijk[0])
    c = np.asarray(fx.cell, dtype=np.float64)
    dij = np.array(minimum_image(c, tuple(x[i] - x[j])))
    dkj = np.array(minimum_image(c, tuple(x[k] - x[j])))
    x[j] = x[j] + 0.5 * (dij + dkj)   # the centre midway between its partners: 180 degrees
    eo = EnergyOptions(cutoff=6.0, skin=1.0, electrostatics="dsf", precision="double")
    ro = RelaxOptions(max_iterations=0, energy=eo, pushoff=False)
    mine = relax(RefEvaluator(ref, fx.ff, eo), x, fx.cell, ro)
    theirs = ref.relax(fx.ff, x, fx.cell, ro)
    assert any("stuck at 180" in n for n in theirs["notes"]) and any("stuck at 180" in n for n in mine["notes"])
    moved = np.linalg.norm(mine["x"] - x, axis=1)
    assert abs(moved[j] - 0.15) < 1e-12 and np.count_nonzero(moved) == 1
    assert np.max(np.abs(mine["x"] - theirs["x"])) < 1e-12


def test_kick_needs_a_bent_angle():
    fx = load("ps_small")
    x = np.array(fx.x, dtype=np.float64)
    assert kick_linear_angles(x, fx.cell, fx.ff, 1) == 0
    assert np.array_equal(x, fx.x)


def _density(ff, cell):
    a, b, c = cell[3:6], cell[6:9], cell[9:12]
    return float(np.sum(ff.mass)) / 6.02214076e23 / (abs(np.dot(a, np.cross(b, c))) * 1e-24)
