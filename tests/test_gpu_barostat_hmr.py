"""The Berendsen barostat (isotropic and per axis) and hydrogen mass repartitioning on the device against the
reference's run_dynamics (oracle/_ref, the reference core built from its sources).

Berendsen scales the cell every barostat_every steps from the pressure of that step (core/src/dynamics.cpp:668-723):
the same factor on every axis, or one per coupled axis from the diagonal of the pressure tensor. Hydrogen mass
repartitioning (dynamics.cpp:125-147) moves mass from each hydrogen's bonded heavy atom to the hydrogen before the run.
Both are deterministic with NVE or Nose-Hoover, so the FP64 device run follows the reference's thermo rows (volume and
pressure included) at the tolerances of the other FP64 dynamics tests.
"""
import math

import numpy as np
import pytest

from caps_b200 import DynamicsOptions, EnergyOptions, Evaluator
from tests.fixtures import load

pytestmark = pytest.mark.gpu


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def _opts(**kw):
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision=kw.pop("precision", "double"))
    base = dict(dt=1.0, steps=30, temperature=300.0, thermostat="none", tau_t=100.0, thermo_every=5, seed=4, energy=eo)
    base.update(kw)
    return DynamicsOptions(**base)


def _compare(rows, ref_rows, tol, keys):
    assert len(rows) == len(ref_rows), (len(rows), len(ref_rows))
    for a, b in zip(rows, ref_rows):
        assert a["step"] == b["step"]
        for k in keys:
            assert abs(a[k] - b[k]) <= tol * max(1.0, abs(b[k])), (a["step"], k, a[k], b[k])


KEYS = ("potential", "kinetic", "total", "volume", "pressure")


@pytest.mark.parametrize("thermostat", ["none", "nose-hoover"])
def test_fp64_berendsen_follows_reference(thermostat):
    ref = _ref()
    fx = load("ps_small")
    o = _opts(thermostat=thermostat, barostat="berendsen", tau_p=100.0, compressibility=4.5e-5, barostat_every=5)
    out = Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    _compare(out["thermo"], r["thermo"], 1e-7, KEYS)
    assert out["thermo"][-1]["volume"] != out["thermo"][0]["volume"]
    np.testing.assert_allclose(out["cell"], r["cell"], rtol=0, atol=1e-9)


def test_fp64_berendsen_per_axis_follows_reference():
    """Per-axis coupling, the y axis held, x driven towards 200 atm and z towards the common target: the cell's
    diagonal follows the reference's, y unchanged."""
    ref = _ref()
    fx = load("ps_small")
    o = _opts(barostat="berendsen", tau_p=100.0, barostat_every=5, anisotropic=True, couple_axis=(True, False, True),
              axis_pressure=(200.0, math.nan, math.nan))
    out = Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    _compare(out["thermo"], r["thermo"], 1e-7, KEYS)
    np.testing.assert_allclose(out["cell"], r["cell"], rtol=0, atol=1e-9)
    c0, c1 = np.asarray(fx.cell, dtype=float).reshape(-1)[3:].reshape(3, 3), np.asarray(out["cell"])[3:].reshape(3, 3)
    assert c1[1, 1] == c0[1, 1] and c1[0, 0] != c0[0, 0] and c1[2, 2] != c0[2, 2]


@pytest.mark.parametrize("barostat", ["berendsen", "c-rescale"])
def test_fp64_barostat_with_constraints_follows_reference(barostat):
    """With SHAKE on C-H the step's constraint virial is carried over a cell rescaling scaled with the cell, as the
    reference does (dynamics.cpp:448-456): the pressure of the rows after a barostat step follows the reference's."""
    ref = _ref()
    fx = load("ps_small")
    o = _opts(thermostat="nose-hoover", barostat=barostat, tau_p=100.0, barostat_every=5, constraints="h-bonds")
    out = Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    _compare(out["thermo"], r["thermo"], 1e-6, KEYS)


def test_fp64_hmr_follows_reference():
    """Hydrogens at 3.024 u (their carbons lighter by the difference) and SHAKE on C-H at 2 fs: the reference's rows and
    positions; the run reports the repartitioning as the reference does, and a later run without it on the same engine
    takes the force field's masses again."""
    ref = _ref()
    fx = load("ps_small")
    o = _opts(dt=2.0, steps=20, thermostat="nose-hoover", constraints="h-bonds", hmr=3.024)
    ev = Evaluator(fx.ff, o.energy)
    out = ev.run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    _compare(out["thermo"], r["thermo"], 1e-6, ("potential", "kinetic", "total", "conserved", "temperature"))
    assert np.max(np.abs(out["x"] - r["x"])) < 1e-6
    assert "hydrogen mass repartitioning: 102 hydrogens at 3.024 u" in out["report"], out["report"]
    plain = _opts(dt=2.0, steps=20, thermostat="nose-hoover", constraints="h-bonds")
    a = ev.run(fx.x, fx.cell, plain)
    b = ref.run(fx.ff, fx.x, fx.cell, plain)
    _compare(a["thermo"], b["thermo"], 1e-6, ("potential", "kinetic", "total"))
    ev.close()


def test_berendsen_mixed_runs_and_rejections():
    """The mixed path takes the Berendsen barostat; per-axis coupling is refused with stochastic cell rescaling, as the
    reference refuses it (dynamics.cpp:84)."""
    fx = load("ps_small")
    o = _opts(precision="mixed", thermostat="nose-hoover", barostat="berendsen", tau_p=100.0, barostat_every=5, steps=50)
    out = Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o)
    assert np.all(np.isfinite(out["x"])) and out["thermo"][-1]["volume"] != out["thermo"][0]["volume"]
    bad = _opts(thermostat="bussi", barostat="c-rescale", anisotropic=True)
    with pytest.raises(Exception, match="per-axis pressure coupling is available with the Berendsen barostat"):
        Evaluator(fx.ff, bad.energy).run(fx.x, fx.cell, bad)
