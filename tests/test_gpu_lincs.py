"""LINCS (constraint_algorithm = "lincs") on the device against the reference's run_dynamics (oracle/_ref, the
reference core built from its sources).

The reference solves the positions with LINCS of order 4 and its rotational corrections (core/src/constraints.cpp:
125-185) and the velocities with RATTLE; the device solves each constraint cluster alone with the same expansion, the
same couplings in the same order and the same iteration rule (constraints of different clusters share no atom, so the
reference's matrix is block-diagonal over them). The clusters stop iterating on their own rather than with the whole
set, so the positions agree to the iteration tolerance (1e-8 relative), and the FP64 thermo rows to the tolerances of
the SHAKE tests.
"""
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


def _compare(rows, ref_rows, tol, keys=("potential", "kinetic", "total", "conserved", "temperature")):
    assert len(rows) == len(ref_rows), (len(rows), len(ref_rows))
    for a, b in zip(rows, ref_rows):
        assert a["step"] == b["step"]
        for k in keys:
            assert abs(a[k] - b[k]) <= tol * max(1.0, abs(b[k])), (a["step"], k, a[k], b[k])


def _opts(**kw):
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision=kw.pop("precision", "double"))
    base = dict(dt=2.0, steps=40, temperature=300.0, thermostat="nose-hoover", tau_t=100.0, thermo_every=10, seed=4,
                constraints="h-bonds", constraint_algorithm="lincs", energy=eo)
    base.update(kw)
    return DynamicsOptions(**base)


def test_fp64_lincs_run_follows_reference():
    """Polystyrene C-H clusters (CH, CH2 and aromatic CH) at 2 fs: the thermo rows and the end positions follow the
    reference's LINCS run; every C-H bond holds its length; the run reports the solver as the reference does."""
    ref = _ref()
    fx = load("ps_small")
    o = _opts()
    out = Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    _compare(out["thermo"], r["thermo"], 1e-6)
    assert np.max(np.abs(out["x"] - r["x"])) < 1e-6
    assert "constraint solver: LINCS (order 4) for positions, RATTLE for velocities" in out["report"], out["report"]
    ff = fx.ff
    h = ff.element == 1
    worst = 0.0
    for (i, j), (k, r0) in zip(ff.bond_ij, ff.bond_k_r0):
        if h[i] or h[j]:
            d = np.linalg.norm(out["x"][j] - out["x"][i])
            worst = max(worst, abs(d - r0) / r0)
    assert worst < 1e-7, worst


def test_fp64_lincs_rigid_water_follows_reference():
    """Rigid SPC/E waters under LINCS: three coupled constraints per water (the device takes them in the general
    cluster layout, not SETTLE, as the reference has no SETTLE); the rows follow the reference's LINCS run."""
    from caps_b200.systems import spce_water
    ref = _ref()
    ff, x, cell = spce_water(216, seed=5)
    eo = EnergyOptions(cutoff=8.0, skin=1.0, electrostatics="pme", pme_order=4, precision="double")
    eq = DynamicsOptions(dt=0.5, steps=400, temperature=300.0, thermostat="langevin", tau_t=20.0, constraints="h-bonds",
                         thermo_every=400, seed=9, energy=eo)
    r0 = ref.run(ff, x, cell, eq)
    o = DynamicsOptions(dt=1.0, steps=20, temperature=300.0, thermostat="none", constraints="h-bonds", constraint_algorithm="lincs",
                        thermo_every=5, seed=9, energy=eo)
    out = Evaluator(ff, eo).run(r0["x"], cell, o, v=r0["v"])
    r = ref.run(ff, r0["x"], cell, o, v=r0["v"])
    _compare(out["thermo"], r["thermo"], 1e-6)
    X = out["x"].reshape(-1, 3, 3)
    d_oh = np.linalg.norm(X[:, 1:] - X[:, :1], axis=2)
    assert np.max(np.abs(d_oh - 1.0)) < 1e-7


def test_lincs_then_shake_on_one_engine_and_mixed():
    """The constraint set is rebuilt when the algorithm changes on the same engine (a SHAKE run after a LINCS run
    follows the reference's SHAKE run), and the mixed path takes LINCS too."""
    ref = _ref()
    fx = load("ps_small")
    o = _opts(steps=20)
    ev = Evaluator(fx.ff, o.energy)
    ev.run(fx.x, fx.cell, o)
    s = _opts(steps=20, constraint_algorithm="shake")
    a = ev.run(fx.x, fx.cell, s)
    b = ref.run(fx.ff, fx.x, fx.cell, s)
    _compare(a["thermo"], b["thermo"], 1e-6)
    assert "LINCS" not in a["report"]
    m = _opts(steps=50, precision="mixed")
    out = Evaluator(fx.ff, m.energy).run(fx.x, fx.cell, m)
    assert np.all(np.isfinite(out["x"]))
