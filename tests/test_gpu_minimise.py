"""Minimisation with the device engine (caps_b200.minimise on an FP64 Evaluator) against the reference's minimise
(core/src/relax.cpp:65, oracle/_ref): the device forces match the reference's to 1e-12, so every method takes the
reference's path (iterations, evaluations) to the same energy. The engine is created once and serves every
evaluation."""
import numpy as np
import pytest

from caps_b200 import EnergyOptions, Evaluator
from caps_b200.minimise import MinimiseOptions, minimise
from tests.fixtures import load

pytestmark = pytest.mark.gpu


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


@pytest.mark.parametrize("method", ["sd", "cg", "lbfgs", "fire"])
def test_device_minimise_follows_reference(method):
    ref = _ref()
    fx = load("ps_small")
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision="double")
    mo = MinimiseOptions(method=method, ftol=1e-4, etol=0.0, max_iterations=40, restraints=[(0, 7, 3.5, 10.0)])
    ev = Evaluator(fx.ff, eo)
    mine = minimise(ev, fx.x, fx.cell, mo)
    theirs = ref.minimise(fx.ff, eo, fx.x, fx.cell, mo)
    assert mine["stopped_by"] == theirs["stopped_by"]
    assert mine["iterations"] == theirs["iterations"] and mine["evaluations"] == theirs["evaluations"]
    assert abs(mine["energy"] - theirs["energy"]) <= 1e-8 * max(1.0, abs(theirs["energy"]))
    assert np.max(np.abs(mine["x"] - theirs["x"])) < 1e-6
    assert ev.list_builds() >= 1


def test_mixed_minimise_lowers_energy():
    fx = load("ps_medium")
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=4, precision="mixed")
    ev = Evaluator(fx.ff, eo)
    e0, _ = ev.compute(fx.x, fx.cell)
    out = minimise(ev, fx.x, fx.cell, MinimiseOptions(method="lbfgs", ftol=0.01, max_iterations=100))
    assert out["iterations"] > 0 and out["energy"] < e0["total"]
