"""Stage chains (caps_b200.equilibrate) against the reference's equilibrate (core/src/equilibrate.cpp:199, oracle/_ref),
and batched replicas against single runs. Each replica keeps one device engine for every stage.

FP64: a short protocol (NVT, NVT with the LJ forces capped, NPT with stochastic cell rescaling, NVE, an NVT ramp) must
give the reference's stage summaries (second-half means of temperature, pressure, density, potential; the density at
the stage's end) to the precision its trajectories follow the reference. Mixed: replicas that differ in seed and
pressure give their single runs' summaries bit for bit."""
import numpy as np
import pytest

from caps_b200 import DynamicsOptions, EnergyOptions, EquilibrateOptions, Evaluator, equilibrate, parse_protocol
from tests.fixtures import load

pytestmark = pytest.mark.gpu

PROTOCOL = """nvt 0.02 ps T 450
nvt 0.01 ps T 300 cap 50
npt 0.02 ps T 400 P 2000 atm
nve 0.01 ps
nvt 0.02 ps T 350 to 420
"""


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def _eq(precision, protocol=PROTOCOL, **md):
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision=precision)
    base = dict(dt=1.0, thermostat="bussi", tau_t=50.0, barostat="c-rescale", tau_p=200.0, seed=13, energy=eo)
    base.update(md)
    return EquilibrateOptions(stages=parse_protocol(protocol), md=DynamicsOptions(**base), thermo_ps=0.005)


def test_fp64_equilibrate_follows_reference():
    ref = _ref()
    fx = load("ps_small")
    eq = _eq("double")
    mine = equilibrate([Evaluator(fx.ff, eq.md.energy)], [fx.x], [fx.cell], [eq])[0]
    theirs = ref.equilibrate(fx.ff, fx.x, fx.cell, eq)
    assert len(mine["stages"]) == len(theirs["stages"]) == 5
    for a, b in zip(mine["stages"], theirs["stages"]):
        assert a["ps"] == pytest.approx(b["ps"], rel=1e-12)
        for k in ("temperature", "pressure", "density", "potential", "density_end"):
            assert abs(a[k] - b[k]) <= 1e-6 * max(1.0, abs(b[k])), (a["label"], k, a[k], b[k])
    assert np.max(np.abs(mine["cell"] - theirs["cell"])) < 1e-6


def test_batched_equilibrate_equals_single_runs():
    proto = "nvt 0.02 ps T 450\nnpt 0.02 ps T 400 P 2000 atm\nnvt 0.02 ps T 350 to 420\n"
    fxs = [load("ps_small"), load("ps_small"), load("ps_medium")]
    eqs = [_eq("mixed", proto, seed=3), _eq("mixed", proto.replace("2000", "500"), seed=8), _eq("mixed", proto, seed=21)]
    single = []
    for fx, eq in zip(fxs, eqs):
        ev = Evaluator(fx.ff, eq.md.energy)
        single.append(equilibrate([ev], [fx.x], [fx.cell], [eq])[0])
        ev.close()
    evs = [Evaluator(fx.ff, eq.md.energy) for fx, eq in zip(fxs, eqs)]
    batch = equilibrate(evs, [fx.x for fx in fxs], [fx.cell for fx in fxs], eqs)
    for a, b in zip(single, batch):
        assert a["stages"] == b["stages"]
        assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["cell"], b["cell"])


def test_equilibrate_rejects_different_stage_lengths():
    fx = load("ps_small")
    a, b = _eq("mixed", "nvt 0.02 ps T 400\n"), _eq("mixed", "nvt 0.03 ps T 400\n")
    evs = [Evaluator(fx.ff, a.md.energy), Evaluator(fx.ff, b.md.energy)]
    with pytest.raises(ValueError):
        equilibrate(evs, [fx.x, fx.x], [fx.cell, fx.cell], [a, b])
