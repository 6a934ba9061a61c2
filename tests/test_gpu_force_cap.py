"""The push-off force cap (EnergyOptions::force_cap, field.cpp:557-581, 1450-1454) on configurations where pairs do come
inside the cap radius: the Kremer-Grest chains before their push-off, and a polystyrene cell with every atom moved at
random by 0.4 Å, in the 12-6 and 9-6 forms, with and without Coulomb. FP64 against the reference at the parity bar,
and the capped dynamics of a push-off (Bussi, Coulomb off) following the reference's thermo rows."""
import dataclasses

import numpy as np
import pytest

from caps_b200 import DynamicsOptions, EnergyOptions, Evaluator
from tests.fixtures import load, rel_rms

pytestmark = pytest.mark.gpu

TERMS = ["bond", "angle", "dihedral", "improper", "vdw", "coulomb"]


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def _check(t, f, rt, rf):
    for k in TERMS:
        assert abs(t[k] - rt[k]) <= 1e-12 * abs(rt[k]) + 1e-9, (k, t[k], rt[k])
    assert abs(t["virial"] - rt["virial"]) <= 1e-11 * abs(rt["virial"]) + 1e-8
    assert rel_rms(f, rf) <= 1e-12, rel_rms(f, rf)


@pytest.mark.parametrize("cap", [5.0, 20.0, 100.0])
def test_capped_kg_chains_match_reference(cap):
    ref = _ref()
    fx = load("kg")
    eo = dataclasses.replace(fx.options(0, "double"), force_cap=cap)
    t, f = Evaluator(fx.ff, eo).compute(fx.x, fx.cell)
    rt, rf = ref.compute(fx.ff, eo, fx.x, fx.cell)
    _check(t, f, rt, rf)
    assert np.abs(rf).max() < 1e6   # the cap holds the overlaps' forces down


@pytest.mark.parametrize("form", ["lj12-6", "lj9-6"])
@pytest.mark.parametrize("coulomb", [True, False])
def test_capped_close_contacts_match_reference(form, coulomb):
    ref = _ref()
    fx = load("ps_small")
    ff = dataclasses.replace(fx.ff, pair_form=form)
    x = fx.x + np.random.default_rng(11).normal(0, 0.4, fx.x.shape)
    eo = EnergyOptions(cutoff=6.0, skin=1.0, electrostatics="pme", pme_order=5, coulomb=coulomb, precision="double", force_cap=5.0)
    t, f = Evaluator(ff, eo).compute(x, fx.cell)
    rt, rf = ref.compute(ff, eo, x, fx.cell)
    _check(t, f, rt, rf)
    t0, _ = ref.compute(ff, dataclasses.replace(eo, force_cap=0.0), x, fx.cell)
    assert t0["vdw"] > rt["vdw"] + 1.0   # pairs are inside the cap radius: the cap lowers their energy


def test_capped_pushoff_dynamics_follow_reference():
    ref = _ref()
    fx = load("ps_small")
    eo = EnergyOptions(cutoff=6.0, skin=1.0, electrostatics="pme", pme_order=5, precision="double")
    soft = dataclasses.replace(eo, force_cap=5.0, coulomb=False)
    md = DynamicsOptions(dt=1.0, steps=20, temperature=300.0, thermostat="bussi", tau_t=100.0, seed=1, thermo_every=2, new_velocities=True,
                         energy=soft)
    ev = Evaluator(fx.ff, eo)
    ev.set_options(soft)   # as relax switches its evaluator to a push-off stage
    out = ev.run(fx.x, fx.cell, md)
    r = ref.run(fx.ff, fx.x, fx.cell, md)
    assert len(out["thermo"]) == len(r["thermo"])
    for a, b in zip(out["thermo"], r["thermo"]):
        for k in ("potential", "kinetic", "conserved"):
            assert abs(a[k] - b[k]) <= 1e-9 * max(1.0, abs(b[k])), (a["step"], k, a[k], b[k])
