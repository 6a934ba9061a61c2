"""The rest of the Evaluator interface (core/include/caps/field.hpp:327-356) against the reference (oracle/_ref):
pairs(), freeze_pairs / unfreeze, reload, threads, and a switch of precision through set_options.

The FP64 bar is the parity bar of the force tests: energy terms to 1e-12 relative (+1e-9 absolute), forces to 1e-12
of the RMS force. A frozen list runs on the FP64 path in both precisions, as the reference's (field.cpp:845).
"""
import dataclasses

import numpy as np
import pytest

from caps_b200 import EnergyOptions, Evaluator, DynamicsOptions
from tests.fixtures import load, rel_rms

pytestmark = pytest.mark.gpu

TERMS = ["bond", "angle", "dihedral", "improper", "vdw", "coulomb"]


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def _same(t, f, rt, rf, tol=1e-12):
    for k in TERMS:
        assert abs(t[k] - rt[k]) <= tol * abs(rt[k]) + 1e-9, (k, t[k], rt[k])
    for c in range(6):
        assert abs(t["w"][c] - rt["w"][c]) <= 10 * tol * abs(rt["virial"]) + 1e-8, ("w", c, t["w"][c], rt["w"][c])
    assert rel_rms(f, rf) <= tol, rel_rms(f, rf)


@pytest.mark.parametrize("name", ["ps_small", "ps_medium", "lj_triclinic", "kg"])
def test_pairs_match_reference(name):
    ref = _ref()
    fx = load(name)
    o = fx.options(0, "double")
    ev = Evaluator(fx.ff, o)
    ev.compute(fx.x, fx.cell)
    assert ev.pairs() == ref.pairs(fx.ff, o, fx.x, fx.cell)
    m = Evaluator(fx.ff, fx.options(0, "mixed"))
    if np.abs(fx.forces[(0, "double")]).max() < 1e9:
        m.compute(fx.x, fx.cell)
    assert m.pairs() == ref.pairs(fx.ff, fx.options(0, "mixed"), fx.x, fx.cell) == 0


def _deformed(x, cell, eps, seed, jiggle):
    """Positions and cell under a small symmetric strain (affine about the origin), plus random moves."""
    rng = np.random.default_rng(seed)
    c = np.asarray(cell, dtype=np.float64).reshape(4, 3)
    e = np.eye(3) + eps * np.array([[1.0, 0.4, -0.2], [0.4, -0.5, 0.3], [-0.2, 0.3, 0.8]])
    y = (np.asarray(x) - c[0]) @ e.T + c[0] + rng.normal(0, jiggle, np.shape(x))
    d = np.vstack([c[0], c[1:] @ e.T])
    return y, d


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("name,electrostatics", [("ps_small", "pme"), ("lj_triclinic", "pme"), ("ps_small", "dsf")])
def test_frozen_pairs_follow_reference(precision, name, electrostatics):
    """Frozen at the fixture, evaluated under a strain of 1e-3 with moves of 0.3 Å (pairs cross the cut-off both
    ways: the frozen ones beyond it take the closed-form Coulomb term)."""
    ref = _ref()
    fx = load(name)
    o = dataclasses.replace(fx.options(0, precision), electrostatics=electrostatics)
    ev = Evaluator(fx.ff, o)
    ev.compute(fx.x, fx.cell)   # a list built before the freeze, as a caller's evaluator has
    ev.freeze_pairs(fx.x, fx.cell)
    for eps, jig, seed in [(1e-3, 0.0, 1), (-1e-3, 0.3, 2), (2e-3, 0.3, 3)]:
        y, d = _deformed(fx.x, fx.cell, eps, seed, jig)
        t, f = ev.compute(y, d)
        rt, rf, npairs = ref.freeze_compute(fx.ff, o, fx.x, fx.cell, y, d)
        _same(t, f, rt, rf)
        assert ev.pairs() == npairs
    with pytest.raises(ValueError, match="frozen"):
        ev.run(fx.x, fx.cell, DynamicsOptions(steps=2, energy=o))
    # unfrozen: the engine's own path again, bit for bit a fresh engine's in mixed precision
    ev.unfreeze()
    y, d = _deformed(fx.x, fx.cell, 1e-3, 7, 0.05)
    t1, f1 = ev.compute(y, d)
    t2, f2 = Evaluator(fx.ff, o).compute(y, d)
    if precision == "mixed":
        assert np.array_equal(f1, f2) and t1["vdw"] == t2["vdw"] and t1["coulomb"] == t2["coulomb"]
    else:
        assert rel_rms(f1, f2) < 1e-13


def _changed(ff):
    """The same atoms with other charges, bond and angle constants, and one dihedral fewer (a topology edit)."""
    return dataclasses.replace(ff, charge=ff.charge * 0.9, bond_k_r0=ff.bond_k_r0 * np.array([1.2, 1.0]),
                               angle_kt_theta0=ff.angle_kt_theta0 * np.array([0.8, 1.0]), dihedral_ijkl=ff.dihedral_ijkl[:-1],
                               dihedral_v_delta=ff.dihedral_v_delta[:-1], dihedral_n=ff.dihedral_n[:-1])


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_reload_follows_reference(precision):
    ref = _ref()
    fx = load("ps_small")
    o = fx.options(0, precision)
    ff2 = _changed(fx.ff)
    ev = Evaluator(fx.ff, o)
    ev.compute(fx.x, fx.cell)
    ev.reload(ff2)
    t, f = ev.compute(fx.x, fx.cell)
    if precision == "double":
        rt, rf = ref.reload_compute(fx.ff, ff2, o, fx.x, fx.cell)
        _same(t, f, rt, rf)
    t2, f2 = Evaluator(ff2, o).compute(fx.x, fx.cell)
    if precision == "mixed":
        assert np.array_equal(f, f2) and t["coulomb"] == t2["coulomb"]
    with pytest.raises(ValueError, match="number of atoms"):
        small = load("kg")
        ev.reload(small.ff)


def test_precision_switch_through_set_options():
    """mixed -> FP64 -> mixed on one engine: each evaluation equals a fresh engine's of that precision."""
    fx = load("ps_medium")
    om, od = fx.options(0, "mixed"), fx.options(0, "double")
    ev = Evaluator(fx.ff, om)
    tm, fm = ev.compute(fx.x, fx.cell)
    ev.set_options(od)
    td, fd = ev.compute(fx.x, fx.cell)
    rd, rfd = Evaluator(fx.ff, od).compute(fx.x, fx.cell)
    _same(td, fd, rd, rfd, tol=1e-13)
    ev.set_options(om)
    tm2, fm2 = ev.compute(fx.x, fx.cell)
    assert np.array_equal(fm, fm2) and tm["vdw"] == tm2["vdw"]


def test_threads_is_the_sm_count():
    import torch
    fx = load("ps_small")
    ev = Evaluator(fx.ff, fx.options(0, "mixed"))
    assert ev.threads() == torch.cuda.get_device_properties(0).multi_processor_count
