"""The class II 9-6 pair form (ForceField::pair_form "lj9-6": eps (2 (s/r)^9 - 3 (s/r)^6), field.cpp:505-506, 1471-1475,
2523-2529) on the device against the reference core (oracle/_ref) on the same cells: FP64 energies and forces at the
FP64 bar (1e-12), with the cut-off shift or the tail correction, 1-4 pairs, PME or damped shifted force, and the
push-off force cap; the mixed path within the mixed tolerances; FP64 dynamics following the reference's rows."""
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


def _ff96(name):
    fx = load(name)
    return fx, dataclasses.replace(fx.ff, pair_form="lj9-6")


@pytest.mark.parametrize("name,elec,tail,cap", [("ps_small", "pme", True, 0.0), ("ps_small", "pme", False, 0.0),
                                                ("lj_triclinic", "dsf", False, 0.0), ("ps_medium", "dsf", True, 0.0),
                                                ("ps_small", "pme", False, 20.0)])
def test_fp64_lj96_matches_reference(name, elec, tail, cap):
    ref = _ref()
    fx, ff = _ff96(name)
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics=elec, pme_order=5, tail=tail, precision="double", force_cap=cap)
    t, f = Evaluator(ff, eo).compute(fx.x, fx.cell)
    rt, rf = ref.compute(ff, eo, fx.x, fx.cell)
    for k in TERMS:
        assert abs(t[k] - rt[k]) <= 1e-12 * abs(rt[k]) + 1e-9, (k, t[k], rt[k])
    assert abs(t["virial"] - rt["virial"]) <= 1e-11 * abs(rt["virial"]) + 1e-8
    if tail:
        assert abs(t["tail_energy"] - rt["tail_energy"]) <= 1e-12 * abs(rt["tail_energy"])
    assert rel_rms(f, rf) <= 1e-12


def test_mixed_lj96_matches_double():
    fx, ff = _ff96("ps_medium")
    eo = dict(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=4, tail=True)
    td, fd = Evaluator(ff, EnergyOptions(precision="double", **eo)).compute(fx.x, fx.cell)
    tm, fm = Evaluator(ff, EnergyOptions(precision="mixed", **eo)).compute(fx.x, fx.cell)
    assert abs(tm["vdw"] - td["vdw"]) <= 2e-6 * abs(td["vdw"]) + 1e-4
    assert rel_rms(fm, fd) <= 5e-6


def test_fp64_lj96_dynamics_follows_reference():
    ref = _ref()
    fx, ff = _ff96("ps_small")
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision="double")
    o = DynamicsOptions(dt=1.0, steps=20, temperature=300.0, thermostat="nose-hoover", tau_t=100.0, thermo_every=5, seed=4, energy=eo)
    out = Evaluator(ff, eo).run(fx.x, fx.cell, o)
    r = ref.run(ff, fx.x, fx.cell, o)
    assert len(out["thermo"]) == len(r["thermo"])
    for a, b in zip(out["thermo"], r["thermo"]):
        for k in ("potential", "kinetic", "conserved"):
            assert abs(a[k] - b[k]) <= 1e-9 * max(1.0, abs(b[k])), (a["step"], k, a[k], b[k])


def test_unknown_pair_form_is_refused():
    fx, _ = _ff96("ps_small")
    with pytest.raises(ValueError):
        Evaluator(dataclasses.replace(fx.ff, pair_form="buckingham"), EnergyOptions(precision="double"))
