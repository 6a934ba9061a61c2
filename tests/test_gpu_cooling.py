"""Stepwise cooling (caps_b200.run_cooling) against the reference's run_cooling (core/src/mechanics.cpp:1381,
oracle/_ref), and batched replicas against single runs.

FP64: one structure through a short ladder (Bussi at each rung, with and without stochastic cell rescaling) must give
the reference's points (rung averages of density and potential energy) to the precision its trajectories follow the
reference (1e-6 relative over ~100 steps). The barostat case also checks that the host random stream is consumed in the
reference's order (each step's thermostat draws, then a barostat step's normal). Mixed: replicas that differ in seed
and pressure, cooled together, give the points of their individual scans bit for bit.
"""
import numpy as np
import pytest

from caps_b200 import CoolingOptions, DynamicsOptions, EnergyOptions, Evaluator, run_cooling
from tests.fixtures import load

pytestmark = pytest.mark.gpu


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def _co(precision, **kw):
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision=precision)
    base = dict(energy=eo, t_start=420.0, t_end=340.0, t_step=20.0, ps_per_step=0.02, equilibrate_ps=0.02, dt=1.0, tau_t=50.0,
                tau_p=200.0, barostat="none", seed=7, new_velocities=True)
    base.update(kw)
    return CoolingOptions(**base)


@pytest.mark.parametrize("barostat", ["none", "c-rescale"])
def test_fp64_cooling_follows_reference(barostat):
    ref = _ref()
    fx = load("ps_small")
    co = _co("double", barostat=barostat)
    ev = Evaluator(fx.ff, co.energy)
    # the Tg fit is the caller's: CAPS passes its own fit_bilinear, here the reference's through the oracle
    mine = run_cooling([ev], [fx.x], [fx.cell], [co], fit=lambda T, y, o: ref.fit_tg(T, y, o.fit, o.glassy_max, o.rubbery_min))[0]
    theirs = ref.run_cooling(fx.ff, fx.x, fx.cell, co)
    assert len(mine["points"]) == len(theirs["points"]) == 5
    for a, b in zip(mine["points"], theirs["points"]):
        assert a["temperature"] == b["temperature"]
        for k in ("density", "potential", "specific_volume"):
            assert abs(a[k] - b[k]) <= 1e-6 * max(1.0, abs(b[k])), (a["temperature"], k, a[k], b[k])
        assert abs(a["density_err"] - b["density_err"]) <= 1e-6 * max(1e-3, abs(b["density_err"]))
    assert np.max(np.abs(mine["cell"] - theirs["cell"])) < 1e-6
    assert np.max(np.abs(mine["x"] - theirs["x"])) < 1e-5
    # the fit saw the points' specific volumes, and gives the reference's Tg to the points' precision
    assert mine["fitted"] == [p["specific_volume"] for p in mine["points"]]
    assert mine["fit"]["ok"] == theirs["fit"]["ok"]
    if theirs["fit"]["ok"]:
        assert abs(mine["fit"]["tg"] - theirs["fit"]["tg"]) <= 1e-3 * abs(theirs["fit"]["tg"])


def test_fp64_npt_run_follows_reference():
    """Bussi + stochastic cell rescaling (dynamics.cpp:699-723) over 40 steps, barostat every 10: thermo rows."""
    ref = _ref()
    fx = load("ps_small")
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision="double")
    o = DynamicsOptions(dt=1.0, steps=40, temperature=350.0, thermostat="bussi", tau_t=50.0, barostat="c-rescale", tau_p=200.0,
                        thermo_every=5, seed=11, energy=eo)
    out = Evaluator(fx.ff, eo).run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    assert len(out["thermo"]) == len(r["thermo"])
    for a, b in zip(out["thermo"], r["thermo"]):
        assert a["step"] == b["step"]
        for k in ("potential", "kinetic", "conserved", "volume", "density", "pressure"):
            assert abs(a[k] - b[k]) <= 1e-7 * max(1.0, abs(b[k])), (a["step"], k, a[k], b[k])


def test_batched_cooling_equals_individual_scans():
    fxs = [load("ps_small"), load("ps_small"), load("ps_medium")]
    opts = [_co("mixed", barostat="c-rescale", seed=3), _co("mixed", barostat="c-rescale", seed=9, pressure=200.0),
            _co("mixed", barostat="c-rescale", seed=5)]
    single = []

    def fit(T, y, o):   # a stand-in for the caller's fit: it records what it was given
        return {"T": list(T), "y": list(y), "method": o.fit}

    for fx, co in zip(fxs, opts):
        ev = Evaluator(fx.ff, co.energy)
        single.append(run_cooling([ev], [fx.x], [fx.cell], [co], fit=fit)[0])
        ev.close()
    evs = [Evaluator(fx.ff, co.energy) for fx, co in zip(fxs, opts)]
    batch = run_cooling(evs, [fx.x for fx in fxs], [fx.cell for fx in fxs], opts, fit=fit)
    for a, b in zip(single, batch):
        assert a["points"] == b["points"]
        assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["cell"], b["cell"])
        assert a["fit"] == b["fit"]
        assert a["fit"]["T"] == [p["temperature"] for p in a["points"]]
    assert run_cooling([evs[0]], [fxs[0].x], [fxs[0].cell], [opts[0]])[0]["fit"] is None


def test_cooling_rejects_different_ladders():
    fx = load("ps_small")
    a, b = _co("mixed"), _co("mixed", t_step=10.0)
    evs = [Evaluator(fx.ff, a.energy), Evaluator(fx.ff, b.energy)]
    with pytest.raises(ValueError):
        run_cooling(evs, [fx.x, fx.x], [fx.cell, fx.cell], [a, b])
