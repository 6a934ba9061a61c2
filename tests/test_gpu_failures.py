"""Failure detection with the fault made on the host: inputs that make a kernel raise a bit of the engine's error word
(no kernel traps, faults or hangs), and the reference's FieldError texts back through the C ABI, compared with the
texts the reference itself throws for the same inputs (oracle/_ref).

* a FENE bond stretched past R0: field.cpp:2157-2159, with r and R0;
* positions that stop being finite during a run: dynamics.cpp:757, with the step;
* a constrained hydrogen placed on its partner: constraints.cpp:219 (the bond turned by more than 90 degrees);
* a cell too small for the cut-off: field.cpp:972;
* non-finite input coordinates, refused before any kernel runs.
After each failure the engine stays usable: the next call on good input succeeds.
"""
import numpy as np
import pytest

from caps_b200 import DynamicsOptions, EnergyOptions, Evaluator, FieldError
from tests.fixtures import load

pytestmark = pytest.mark.gpu


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def _ref_text(fn) -> str:
    try:
        fn()
    except RuntimeError as e:
        return str(e)
    raise AssertionError("the reference did not fail")


def _pme(prec="double"):
    return EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision=prec)


@pytest.mark.parametrize("prec", ["double", "mixed"])
def test_fene_overstretch_gives_the_reference_text(prec):
    ref = _ref()
    fx = load("kg")
    x = fx.x.copy()
    d = x[0] - x[1]
    x[0] = x[1] + 1.6 * d / np.linalg.norm(d)   # the chain's end bond at 1.6 sigma, past R0 = 1.5
    want = _ref_text(lambda: ref.compute(fx.ff, fx.options(0, "double"), x, fx.cell))
    assert "stretched to r = 1.600000 Å, past R0 = 1.500000 Å" in want
    ev = Evaluator(fx.ff, fx.options(0, prec))
    with pytest.raises(FieldError) as ei:
        ev.compute(x, fx.cell)
    assert str(ei.value) == want
    # the engine stays usable
    t, f = ev.compute(fx.x, fx.cell) if prec == "double" else (None, None)
    if prec == "double":
        assert np.all(np.isfinite(f))


@pytest.mark.parametrize("thermostat", ["none", "bussi"])
def test_unstable_run_gives_the_reference_text_and_step(thermostat):
    ref = _ref()
    fx = load("ps_small")
    v = np.zeros_like(fx.x)
    v[0, 0] = np.nan        # atom 0 is one the reference checks every step
    o = DynamicsOptions(dt=1.0, steps=12, thermostat=thermostat, temperature=300.0, thermo_every=4, seed=3, energy=_pme())
    want = _ref_text(lambda: ref.run(fx.ff, fx.x, fx.cell, o, v=v))
    assert want.startswith("the simulation became unstable at step 1;")
    ev = Evaluator(fx.ff, o.energy)
    with pytest.raises(FieldError) as ei:
        ev.run(fx.x, fx.cell, o, v=v)
    assert str(ei.value) == want
    out = ev.run(fx.x, fx.cell, o, v=np.zeros_like(fx.x))   # a good run on the same engine afterwards
    assert np.all(np.isfinite(out["x"]))


def test_langevin_unstable_step_is_the_step_it_happened_at():
    fx = load("ps_small")
    v = np.zeros_like(fx.x)
    v[3, 1] = np.inf
    o = DynamicsOptions(dt=1.0, steps=8, thermostat="langevin", temperature=300.0, thermo_every=8, seed=3, energy=_pme())
    with pytest.raises(FieldError, match="became unstable at step 1;"):
        Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o, v=v)


def test_constrained_hydrogen_on_its_partner_gives_the_reference_text():
    ref = _ref()
    fx = load("ps_small")
    h, c = 8, 0          # a C-H bond of the cell (atoms 0 and 8)
    assert fx.ff.element[h] == 1
    x = fx.x.copy()
    x[h] = x[c]
    o = DynamicsOptions(dt=1.0, steps=5, thermostat="none", thermo_every=5, constraints="h-bonds", seed=3, energy=_pme())
    want = _ref_text(lambda: ref.run(fx.ff, x, fx.cell, o))
    ev = Evaluator(fx.ff, o.energy)
    with pytest.raises(FieldError) as ei:
        ev.run(x, fx.cell, o)
    assert str(ei.value) == want == "a constrained bond turned by more than 90° in one step; lower the time step or relax first"
    assert np.all(np.isfinite(ev.run(fx.x, fx.cell, o)["x"]))


@pytest.mark.parametrize("prec", ["double", "mixed"])
def test_cell_too_small_gives_the_reference_text(prec):
    ref = _ref()
    fx = load("ps_small")
    c = fx.cell.copy()
    c[3:] *= 0.02
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="dsf", precision="double")
    want = _ref_text(lambda: ref.compute(fx.ff, eo, fx.x * 0.02, c))
    ev = Evaluator(fx.ff, EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="dsf", precision=prec))
    with pytest.raises(FieldError) as ei:
        ev.compute(fx.x * 0.02, c)
    assert str(ei.value) == want
    t, f = ev.compute(fx.x, fx.cell)
    assert np.all(np.isfinite(f))


def test_non_finite_input_coordinates_are_refused():
    fx = load("ps_small")
    x = fx.x.copy()
    x[5, 2] = np.nan
    ev = Evaluator(fx.ff, _pme())
    with pytest.raises(FieldError, match="non-finite coordinates: atom 6"):
        ev.compute(x, fx.cell)
    assert np.all(np.isfinite(ev.compute(fx.x, fx.cell)[1]))
