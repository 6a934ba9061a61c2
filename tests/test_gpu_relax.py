"""The relaxation stage chain (caps_b200.relax) on a device engine against the reference's relax (relax.cpp:343): in
FP64 the device takes the reference's path (the same stages, stops and iteration counts; energies, densities and
pressures to 1e-7), push-off dynamics under a ramped force cap included; in mixed precision the capped stages run on
the FP64 path, as the reference's, and the chain ends below the force tolerance."""
import numpy as np
import pytest

from caps_b200 import EnergyOptions, Evaluator, RelaxOptions, relax
from tests.fixtures import load

pytestmark = pytest.mark.gpu


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def _density(ff, cell):
    a, b, c = cell[3:6], cell[6:9], cell[9:12]
    return float(np.sum(ff.mass)) / 6.02214076e23 / (abs(np.dot(a, np.cross(b, c))) * 1e-24)


def test_fp64_relax_follows_reference():
    ref = _ref()
    fx = load("ps_small")
    eo = EnergyOptions(cutoff=6.0, skin=1.0, electrostatics="pme", pme_order=5, precision="double")
    c = np.asarray(fx.cell, dtype=np.float64)
    ro = RelaxOptions(method="lbfgs", ftol=0.5, max_iterations=15, energy=eo, pushoff_ramp_ps=0.02, pushoff_ramp_segments=2,
                      target_density=1.05 * _density(fx.ff, c), compress_step=0.05, relax_box=True, pressure=1.0, pressure_tol=500.0,
                      box_cycles=2)
    mine = relax(Evaluator(fx.ff, eo), fx.x, fx.cell, ro)
    theirs = ref.relax(fx.ff, fx.x, fx.cell, ro)
    assert [s["name"] for s in mine["stages"]] == [s["name"] for s in theirs["stages"]]
    for a, b in zip(mine["stages"], theirs["stages"]):
        assert a["stopped_by"] == b["stopped_by"] and a["iterations"] == b["iterations"], (a, b)
        for k in ("energy", "density", "pressure"):
            assert abs(a[k] - b[k]) <= 1e-7 * max(1.0, abs(b[k])), (a["name"], k, a[k], b[k])
    assert mine["evaluations"] == theirs["evaluations"] and mine["converged"] == theirs["converged"]
    assert abs(mine["density_final"] - theirs["density_final"]) <= 1e-9 * theirs["density_final"]
    assert np.max(np.abs(mine["x"] - theirs["x"])) < 1e-5


def test_mixed_relax_reaches_the_force_tolerance():
    fx = load("ps_medium")
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=4, precision="mixed")
    ro = RelaxOptions(method="lbfgs", ftol=2.0, max_iterations=500, energy=eo)
    ev = Evaluator(fx.ff, eo)
    out = relax(ev, fx.x, fx.cell, ro)
    assert out["converged"] and out["fmax_final"] < 2.0
    assert [s["name"] for s in out["stages"]][:4] == ["push-off, force cap 5", "push-off, force cap 20", "push-off, force cap 100",
                                                      "push-off, force cap 500"]
    t, f = ev.compute(out["x"], out["cell"])   # the engine is back on its own (mixed) options
    assert abs(t["total"] - out["final"]["total"]) <= 1e-6 * abs(out["final"]["total"])
