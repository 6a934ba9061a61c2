"""Size-independent properties of the device forces, checked at the benchmark's full size (the 32,000-atom
polystyrene PME melt) where the oracle would take minutes, and on a fixture cell: the reference's own self-consistency
tests of Evaluator (tests/test_relax.cpp:95-170) on the device path.

* forces are minus the energy gradient: central differences, h = 1e-5 Å, within 2e-4 relative (test_relax.cpp:95-118);
* the virial tensor is minus the strain derivative of the energy, every component, sheared strains included
  (test_relax.cpp:142-155), with the tail correction off (its pressure is not the derivative of the truncated energy);
* the energy is periodic: a molecule moved by lattice vectors leaves it unchanged (test_relax.cpp:157-168);
* the mixed path is bit-reproducible at full size, and agrees with FP64 there within the target error.
"""
import numpy as np
import pytest

from caps_b200 import Evaluator
from tests.fixtures import load, ps32k, ps32k_options, rel_rms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    return ps32k()


def _total(t):
    return t["bond"] + t["angle"] + t["dihedral"] + t["improper"] + t["vdw"] + t["coulomb"]


def _fd_forces(ev, x, cell, idx, h=1e-5):
    worst = 0.0
    t, f = ev.compute(x, cell)
    f = f.reshape(-1)
    for k in idx:
        xp, xm = x.copy().reshape(-1), x.copy().reshape(-1)
        xp[k] += h
        xm[k] -= h
        ep = _total(ev.compute(xp, cell)[0])
        em = _total(ev.compute(xm, cell)[0])
        fd = -(ep - em) / (2 * h)
        worst = max(worst, abs(fd - f[k]) / max(1.0, abs(f[k])))
    return worst


def test_fp64_forces_are_the_energy_gradient_at_full_size(big):
    ff, x, _, cell = big
    ev = Evaluator(ff, ps32k_options("double"))
    idx = np.random.default_rng(3).choice(x.size, 24, replace=False)
    assert _fd_forces(ev, x, cell, idx) < 2e-4


def test_fp64_forces_are_the_energy_gradient_on_a_triclinic_cell():
    fx = load("lj_triclinic")
    rng = np.random.default_rng(5)
    x = fx.x + rng.normal(0, 0.02, fx.x.shape)
    ev = Evaluator(fx.ff, fx.options(0, "double"))
    assert _fd_forces(ev, x, fx.cell, rng.choice(x.size, 30, replace=False)) < 2e-4


def _strain_derivative(ev, x, cell, h=1e-6):
    """-dE/d(eps) for the six symmetric strains (xx yy zz xy xz yz), affine about the cell's origin."""
    c = np.asarray(cell, dtype=np.float64).reshape(4, 3)
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    out = []
    for a, b in pairs:
        e = []
        for sg in (1, -1):
            S = np.zeros((3, 3))
            if a == b:
                S[a, a] = sg * h
            else:
                S[a, b] = S[b, a] = 0.5 * sg * h
            F = np.eye(3) + S
            y = (x - c[0]) @ F.T + c[0]
            d = np.vstack([c[0], c[1:] @ F.T])
            e.append(_total(ev.compute(y, d)[0]))
        out.append(-(e[0] - e[1]) / (2 * h))
    return np.array(out)


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_virial_tensor_is_the_strain_derivative_at_full_size(big, precision):
    ff, x, _, cell = big
    ev = Evaluator(ff, ps32k_options(precision, tail=False))
    t, _ = ev.compute(x, cell)
    w = np.array(t["w"])
    assert abs(w[:3].sum() - t["virial"]) <= 1e-9 * abs(t["virial"]) + 1e-9
    d = _strain_derivative(ev, x, cell, h=1e-6 if precision == "double" else 1e-5)
    assert np.all(np.abs(w - d) <= 2e-3 * max(1.0, abs(t["virial"]))), (w, d)


def test_energy_is_periodic_at_full_size(big):
    """The first chain (800 atoms) moved by a - 2c: energy and forces unchanged, in both precisions."""
    ff, x, _, cell = big
    c = np.asarray(cell).reshape(4, 3)
    y = x.copy()
    y[:800] += c[1] - 2 * c[3]
    for precision, tol in (("double", 1e-9), ("mixed", 1e-6)):
        ev = Evaluator(ff, ps32k_options(precision))
        t0, f0 = ev.compute(x, cell)
        t1, f1 = Evaluator(ff, ps32k_options(precision)).compute(y, cell)
        assert abs(_total(t1) - _total(t0)) <= tol * abs(_total(t0)), (precision, _total(t0), _total(t1))
        assert rel_rms(f1, f0) < (1e-9 if precision == "double" else 1e-5)


def test_mixed_at_full_size_is_reproducible_and_within_target(big):
    ff, x, _, cell = big
    a = Evaluator(ff, ps32k_options("mixed"))
    t1, f1 = a.compute(x, cell)
    t2, f2 = Evaluator(ff, ps32k_options("mixed")).compute(x, cell)
    assert np.array_equal(f1, f2) and t1["coulomb"] == t2["coulomb"] and t1["vdw"] == t2["vdw"]
    td, fd = Evaluator(ff, ps32k_options("double")).compute(x, cell)
    assert rel_rms(f1, fd) <= 5e-6
    assert abs(_total(t1) - _total(td)) <= 1e-6 * abs(_total(td))
