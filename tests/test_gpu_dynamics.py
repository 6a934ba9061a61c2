"""Device MD against the reference's run_dynamics (oracle/_ref, the reference core built from its sources).

With the same seed both draw the same initial velocities (the reference's own random stream is reproduced on the
host), and NVE, Nose-Hoover and Bussi runs are deterministic, so the FP64 device run must follow the reference's
thermo rows step by step (to 1e-9 relative over tens of steps; SHAKE's 1e-8 tolerance bounds the constrained runs).
Stochastic thermostats are checked statistically; the mixed path by energy conservation (tests/test_nbnxm.cpp:101-124).
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


def _opts(**kw):
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision=kw.pop("precision", "double"))
    base = dict(dt=1.0, steps=20, temperature=300.0, thermostat="none", tau_t=100.0, thermo_every=5, seed=4, energy=eo)
    base.update(kw)
    return DynamicsOptions(**base)


def _compare(rows, ref_rows, tol, keys=("potential", "kinetic", "total", "conserved", "temperature")):
    assert len(rows) == len(ref_rows), (len(rows), len(ref_rows))
    for a, b in zip(rows, ref_rows):
        assert a["step"] == b["step"]
        for k in keys:
            assert abs(a[k] - b[k]) <= tol * max(1.0, abs(b[k])), (a["step"], k, a[k], b[k])


@pytest.mark.parametrize("thermostat", ["none", "nose-hoover", "bussi"])
def test_fp64_run_follows_reference(thermostat):
    ref = _ref()
    fx = load("ps_small")
    o = _opts(thermostat=thermostat)
    ev = Evaluator(fx.ff, o.energy)
    out = ev.run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    _compare(out["thermo"], r["thermo"], 1e-9)
    assert np.max(np.abs(out["x"] - r["x"])) < 1e-8


@pytest.mark.parametrize("thermostat", ["none", "bussi"])
def test_fp64_respa_run_follows_reference(thermostat):
    """r-RESPA (dynamics.cpp:643-657): bonded forces at dt / 3, non-bonded ones at dt; the reference's thermo rows."""
    ref = _ref()
    fx = load("ps_small")
    o = _opts(thermostat=thermostat, respa=3, dt=1.5, steps=20)
    ev = Evaluator(fx.ff, o.energy)
    out = ev.run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    _compare(out["thermo"], r["thermo"], 1e-9)
    assert np.max(np.abs(out["x"] - r["x"])) < 1e-8


def test_fp64_respa_with_cell_rescaling_follows_reference():
    """r-RESPA (bonded forces at dt / 2) with the Bussi thermostat and stochastic cell rescaling every 5 steps, as the
    reference allows them together (dynamics.cpp:90-94): its thermo rows, volume included."""
    ref = _ref()
    fx = load("ps_small")
    o = _opts(thermostat="bussi", respa=2, dt=1.5, steps=30, barostat="c-rescale", tau_p=200.0, barostat_every=5, thermo_every=5)
    out = Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    _compare(out["thermo"], r["thermo"], 1e-7, keys=("potential", "kinetic", "conserved", "volume", "pressure"))
    assert out["thermo"][-1]["volume"] != out["thermo"][0]["volume"]


def test_pme_split_with_cell_rescaling_runs_npt():
    """The PME split (PME every 2 fs) with Bussi and stochastic cell rescaling, the composite configuration's
    integrator: the cell moves, the temperature holds near its target and the state stays finite."""
    fx = load("ps_medium")
    eo = EnergyOptions(cutoff=10.0, skin=2.0, electrostatics="pme", pme_order=4, precision="mixed")
    o = DynamicsOptions(dt=2.0, steps=300, temperature=350.0, thermostat="bussi", tau_t=50.0, barostat="c-rescale", tau_p=500.0,
                        barostat_every=10, respa=2, respa_split="pme", thermo_every=50, seed=5, energy=eo, new_velocities=True)
    out = Evaluator(fx.ff, eo).run(fx.x, fx.cell, o)
    vols = [r["volume"] for r in out["thermo"]]
    assert len(set(vols)) > 1 and np.all(np.isfinite(out["x"]))
    assert abs(np.mean([r["temperature"] for r in out["thermo"][2:]]) - 350.0) < 40.0


def test_pme_respa_split_conserves_energy():
    """The PME split (the reciprocal sum once per 2 fs outer step, every other term every 1 fs): no reference has it, so
    it must start from the plain run's step-0 row and conserve the total energy about as well as velocity Verlet at 1 fs."""
    fx = load("ps_small")
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision="double")
    common = dict(temperature=300.0, thermostat="none", thermo_every=10, seed=4, energy=eo)
    a = Evaluator(fx.ff, eo).run(fx.x, fx.cell, DynamicsOptions(dt=1.0, steps=400, **common))
    b = Evaluator(fx.ff, eo).run(fx.x, fx.cell, DynamicsOptions(dt=2.0, steps=200, respa=2, respa_split="pme", **common))
    for k in ("potential", "kinetic"):
        assert abs(a["thermo"][0][k] - b["thermo"][0][k]) <= 1e-12 * abs(a["thermo"][0][k])
    ea = np.array([r["total"] for r in a["thermo"]])
    eb = np.array([r["total"] for r in b["thermo"]])
    assert np.std(eb) < 3 * max(np.std(ea), 1e-7 * abs(ea.mean())), (np.std(ea), np.std(eb))


def test_fp64_rigid_water_settle_follows_reference_shake():
    """Rigid SPC/E waters: the device solves them with SETTLE (exact distances), the reference with SHAKE (1e-8 relative
    tolerance); from the same equilibrated state the thermo rows agree to SHAKE's tolerance."""
    from caps_b200.systems import spce_water
    ref = _ref()
    ff, x, cell = spce_water(216, seed=5)
    eo = EnergyOptions(cutoff=8.0, skin=1.0, electrostatics="pme", pme_order=4, precision="double")
    eq = DynamicsOptions(dt=0.5, steps=400, temperature=300.0, thermostat="langevin", tau_t=20.0, constraints="h-bonds",
                         thermo_every=400, seed=9, energy=eo)
    r0 = ref.run(ff, x, cell, eq)
    o = DynamicsOptions(dt=1.0, steps=20, temperature=300.0, thermostat="none", constraints="h-bonds", thermo_every=5, seed=9,
                        energy=eo)
    ev = Evaluator(ff, eo)
    out = ev.run(r0["x"], cell, o, v=r0["v"])
    r = ref.run(ff, r0["x"], cell, o, v=r0["v"])
    _compare(out["thermo"], r["thermo"], 1e-6)
    X = out["x"].reshape(-1, 3, 3)
    d_oh = np.linalg.norm(X[:, 1:] - X[:, :1], axis=2)
    d_hh = np.linalg.norm(X[:, 2] - X[:, 1], axis=1)
    assert np.max(np.abs(d_oh - 1.0)) < 1e-10
    assert np.max(np.abs(d_hh - 2 * np.sin(np.radians(109.47) / 2))) < 1e-10


def test_fp64_shake_run_follows_reference():
    ref = _ref()
    fx = load("ps_small")
    o = _opts(thermostat="nose-hoover", constraints="h-bonds", dt=2.0, steps=40, thermo_every=10)
    ev = Evaluator(fx.ff, o.energy)
    out = ev.run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    _compare(out["thermo"], r["thermo"], 1e-6)
    # every C-H bond at its length
    ff = fx.ff
    h = ff.element == 1
    for (i, j), (k, r0) in zip(ff.bond_ij, ff.bond_k_r0):
        if h[i] or h[j]:
            d = out["x"][j] - out["x"][i]
            assert abs(np.linalg.norm(d) - r0) < 1e-6


def test_mixed_nve_conserves_energy_like_double():
    fx = load("ps_small")
    bands = {}
    for prec in ("double", "mixed"):
        o = _opts(precision=prec, steps=2000, thermo_every=100)
        ev = Evaluator(fx.ff, o.energy)
        out = ev.run(fx.x, fx.cell, o)
        c = [row["conserved"] for row in out["thermo"]]
        bands[prec] = max(c) - min(c)
    assert bands["mixed"] < 1.5 * bands["double"] + 0.05, bands


def test_langevin_holds_temperature():
    fx = load("ps_medium")
    eo = EnergyOptions(cutoff=10.0, electrostatics="pme", pme_order=4, precision="mixed")
    o = DynamicsOptions(dt=1.0, steps=3000, temperature=400.0, thermostat="langevin", tau_t=50.0, thermo_every=100, seed=9, energy=eo)
    out = Evaluator(fx.ff, eo).run(fx.x, fx.cell, o)
    t = np.array([r["temperature"] for r in out["thermo"][10:]])
    assert abs(t.mean() - 400.0) < 12.0, t.mean()
