"""Replicas in lock step (caps_gpu_run_batch) against the same replicas run one by one.

The mixed path sums every force in fixed point, so a replica's trajectory does not depend on what runs beside it: the
batched thermo rows and end states must equal the individual runs' bit for bit. The replicas differ in size, force field
and thermostat settings, as the rungs of a cooling ladder do.
"""
import numpy as np
import pytest

from caps_b200 import DynamicsOptions, EnergyOptions, Evaluator, run_batch
from tests.fixtures import load

pytestmark = pytest.mark.gpu


def _replicas():
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=4, precision="mixed")
    cases = [("ps_small", dict(thermostat="langevin", temperature=500.0, tau_t=100.0)),
             ("ps_medium", dict(thermostat="nose-hoover", temperature=400.0, tau_t=100.0, constraints="h-bonds")),
             ("lj_triclinic", dict(thermostat="bussi", temperature=300.0, tau_t=50.0)),
             ("ps_small", dict(thermostat="bussi", temperature=350.0, tau_t=50.0, seed=5))]
    out = []
    for name, kw in cases:
        fx = load(name)
        o = DynamicsOptions(dt=1.0, steps=60, thermo_every=20, energy=eo, **{"seed": 3, **kw})
        out.append((fx, o))
    return out


def test_batch_equals_individual_runs():
    reps = _replicas()
    single = []
    for fx, o in reps:
        ev = Evaluator(fx.ff, o.energy)
        single.append(ev.run(fx.x, fx.cell, o))
        ev.close()
    evs = [Evaluator(fx.ff, o.energy) for fx, o in reps]
    batch = run_batch(evs, [fx.x for fx, _ in reps], [fx.cell for fx, _ in reps], [o for _, o in reps])
    for r, (a, b) in enumerate(zip(single, batch)):
        assert len(a["thermo"]) == len(b["thermo"]) == 4
        for ra, rb in zip(a["thermo"], b["thermo"]):
            for k in ("potential", "kinetic", "conserved"):
                assert ra[k] == rb[k], (r, ra["step"], k, ra[k], rb[k])
        assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["v"], b["v"]), r
    for ev in evs:
        ev.close()


def test_batch_rejects_unequal_steps():
    fx = load("ps_small")
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", precision="mixed")
    evs = [Evaluator(fx.ff, eo), Evaluator(fx.ff, eo)]
    opts = [DynamicsOptions(steps=10, thermostat="none", energy=eo), DynamicsOptions(steps=20, thermostat="none", energy=eo)]
    with pytest.raises(Exception, match="same number of steps"):
        run_batch(evs, [fx.x, fx.x], [fx.cell, fx.cell], opts)
    for ev in evs:
        ev.close()
