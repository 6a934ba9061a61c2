"""The generic FP64 pair forms (ForceField::pair_func: Buckingham, Morse, Rydberg, SDK, lj/gromacs, cosine-squared with
and without WCA, tabulated; each with an optional cut-off of its own; field.cpp:478-487, 528-555, 1381-1455, 1482-1492,
2508-2522) on the device against the reference core (oracle/_ref) on
the same cells: energies, virial and forces at the FP64 bar (1e-12), with the cut-off shift or the tail correction,
in the non-bonded pairs and the 1-4 pairs, under PME and damped shifted force. A force field with any of them runs the
FP64 path whatever precision is asked for, as the reference's mixed path falls back to its FP64 pair loop."""
import dataclasses

import numpy as np
import pytest

from caps_b200 import EnergyOptions, Evaluator
from tests.fixtures import load, rel_rms

pytestmark = pytest.mark.gpu
TERMS = ["bond", "angle", "dihedral", "improper", "vdw", "coulomb"]


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


# per fixture: Buckingham on a carbon pair (its 1-4 pairs included), Morse with a cut-off of its own, Rydberg
FORMS = {
    "ps_small": {(0, 1): ("buckingham", 30000.0, 0.28, 600.0), (1, 1): ("morse", 0.1, 1.2, 3.8, 6.5),
                 (2, 3): ("rydberg", 50.0, 0.35, -10.0)},
    "lj_triclinic": {(0, 0): ("buckingham", 25000.0, 0.27, 500.0), (1, 2): ("morse", 0.12, 1.1, 3.6, 6.0),
                     (0, 2): ("rydberg", 40.0, 0.3, -5.0, 7.0)},
}


def _table():
    """A tabulated H-H pair from 1.5 Å by 0.01 Å (700 points): a 12-6 well at 2.5 Å and its force -dE/dr."""
    r = 1.5 + 0.01 * np.arange(700)
    e = 0.02 * ((2.5 / r) ** 12 - 2 * (2.5 / r) ** 6)
    f = 0.02 * (12 * 2.5 ** 12 / r ** 13 - 12 * 2.5 ** 6 / r ** 7)
    return (1.5, 0.01, e, f)


# the coarse-grained forms on the polystyrene cell: SDK, lj/gromacs, cosine-squared (with and without WCA), a table
CG = {(0, 0): ("sdk12-4", 0.1, 3.2), (0, 2): ("sdk9-6", 0.05, 2.9), (0, 3): ("sdk12-6", 0.04, 2.9), (1, 2): ("sdk12-5", 0.05, 3.0),
      (1, 3): ("lj/gromacs", 0.03, 2.6), (2, 2): ("cos2", 0.05, 2.5, 5.0), (2, 3): ("cos2-wca", 0.04, 2.6, 4.5),
      (3, 3): ("table", 0, 0, 0)}


def _ff(name):
    if name == "ps_cg":   # every spec as (form, a, b, c)
        fx = load("ps_small")
        return fx, dataclasses.replace(fx.ff, pair_func={k: v + (0.0,) * (4 - len(v)) for k, v in CG.items()}, lj_inner=6.0, tables=[_table()])
    fx = load(name)
    return fx, dataclasses.replace(fx.ff, pair_func=FORMS[name])


@pytest.mark.parametrize("name,elec,tail", [("ps_small", "pme", False), ("ps_small", "pme", True), ("ps_small", "dsf", False),
                                            ("lj_triclinic", "dsf", False), ("lj_triclinic", "dsf", True),
                                            ("ps_cg", "pme", False), ("ps_cg", "dsf", True)])
def test_fp64_pair_forms_match_reference(name, elec, tail):
    ref = _ref()
    fx, ff = _ff(name)
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics=elec, pme_order=5, tail=tail, precision="double")
    t, f = Evaluator(ff, eo).compute(fx.x, fx.cell)
    rt, rf = ref.compute(ff, eo, fx.x, fx.cell)
    for k in TERMS:
        assert abs(t[k] - rt[k]) <= 1e-12 * abs(rt[k]) + 1e-9, (k, t[k], rt[k])
    assert abs(t["virial"] - rt["virial"]) <= 1e-11 * abs(rt["virial"]) + 1e-8
    if tail:
        assert abs(t["tail_energy"] - rt["tail_energy"]) <= 1e-12 * abs(rt["tail_energy"]) + 1e-12
    assert rel_rms(f, rf) <= 1e-12
    # the forms change the answer: the plain LJ force field gives another vdW energy
    t0, _ = Evaluator(fx.ff, eo).compute(fx.x, fx.cell)
    assert abs(t0["vdw"] - t["vdw"]) > 1e-6 * abs(t["vdw"])


def test_pair_forms_run_fp64_when_mixed_is_asked():
    fx, ff = _ff("ps_small")
    eo = dict(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5)
    td, fd = Evaluator(ff, EnergyOptions(precision="double", **eo)).compute(fx.x, fx.cell)
    tm, fm = Evaluator(ff, EnergyOptions(precision="mixed", **eo)).compute(fx.x, fx.cell)
    assert abs(tm["vdw"] - td["vdw"]) <= 1e-12 * abs(td["vdw"])
    assert rel_rms(fm, fd) <= 1e-13


def test_unsupported_pair_form_is_refused():
    fx = load("ps_small")
    with pytest.raises(ValueError, match="unknown pair form"):
        dataclasses.replace(fx.ff, pair_func={(0, 0): ("soft", 0, 0, 0)}).to_struct()
    with pytest.raises(Exception, match="unknown pair form 99"):
        Evaluator(dataclasses.replace(fx.ff, pair_func={(0, 0): (99, 0.1, 3.4, 0.0)}), EnergyOptions(precision="double"))
    with pytest.raises(Exception, match="a table that is not there"):
        Evaluator(dataclasses.replace(fx.ff, pair_func={(0, 0): ("table", 2, 0, 0)}), EnergyOptions(precision="double"))
    with pytest.raises(Exception, match="inner radius below the cut-off"):
        Evaluator(dataclasses.replace(fx.ff, pair_func={(0, 0): ("lj/gromacs", 0.1, 3.4, 0.0)}), EnergyOptions(precision="double"))


@pytest.mark.parametrize("name,elec", [("ps_small", "pme"), ("ps_small", "dsf"), ("lj_triclinic", "dsf")])
def test_fp64_charmm_force_switch_matches_reference(name, elec):
    """ForceField::lj_fsw: every 12-6 pair (the 1-4 pairs too) switched from lj_inner to the cut-off, no shift and no
    tail (field.cpp:440-443, 1455-1469, 2033); the FP64 path whatever precision is asked for."""
    ref = _ref()
    fx = load(name)
    ff = dataclasses.replace(fx.ff, lj_fsw=True, lj_inner=6.5)
    for prec in ("double", "mixed"):
        eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics=elec, pme_order=5, tail=True, precision=prec)
        t, f = Evaluator(ff, eo).compute(fx.x, fx.cell)
        rt, rf = ref.compute(ff, eo, fx.x, fx.cell)
        for k in TERMS:
            assert abs(t[k] - rt[k]) <= 1e-12 * abs(rt[k]) + 1e-9, (prec, k, t[k], rt[k])
        assert abs(t["virial"] - rt["virial"]) <= 1e-11 * abs(rt["virial"]) + 1e-8
        assert t["tail_energy"] == 0.0
        assert rel_rms(f, rf) <= 1e-12
    with pytest.raises(Exception, match="inner radius below the cut-off"):
        Evaluator(dataclasses.replace(fx.ff, lj_fsw=True, lj_inner=9.0), EnergyOptions(cutoff=8.0, precision="double"))
