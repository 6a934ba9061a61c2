"""The MTK barostat (Barostat::MTK: isotropic Martyna-Tobias-Klein pressure coupling with its Nose-Hoover chain, as
LAMMPS fix npt / nph; core/src/dynamics.cpp:479-570, 628-642) on the device against the reference's run_dynamics
(oracle/_ref, the reference core built from its sources).

Every MTK step runs on the host's schedule (the cell moves twice a step): the barostat's chain, the particles' chain
with Nose-Hoover, the volume's momentum from the kinetic energy and the last virial, the remaps of the cell and the
positions about the cell's centre, and the forces with energies and virial. The FP64 rows (volume, pressure and the
extended system's conserved energy included) follow the reference's at the tolerances of the other FP64 dynamics
tests.
"""
import numpy as np
import pytest

from caps_b200 import DynamicsOptions, EnergyOptions, Evaluator
from tests.fixtures import load

pytestmark = pytest.mark.gpu
KEYS = ("potential", "kinetic", "total", "conserved", "volume", "pressure")


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def _opts(**kw):
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="pme", pme_order=5, precision=kw.pop("precision", "double"))
    base = dict(dt=0.5, steps=30, temperature=300.0, thermostat="nose-hoover", tau_t=50.0, barostat="mtk", pressure=1.0,
                tau_p=200.0, thermo_every=5, seed=4, energy=eo)
    base.update(kw)
    return DynamicsOptions(**base)


def _compare(rows, ref_rows, tol, keys=KEYS):
    assert len(rows) == len(ref_rows), (len(rows), len(ref_rows))
    for a, b in zip(rows, ref_rows):
        assert a["step"] == b["step"]
        for k in keys:
            assert abs(a[k] - b[k]) <= tol * max(1.0, abs(b[k])), (a["step"], k, a[k], b[k])


@pytest.mark.parametrize("thermostat", ["nose-hoover", "none"])
def test_fp64_mtk_follows_reference(thermostat):
    """NPT (Nose-Hoover + MTK) and NPH (MTK alone): the rows, the end cell and the positions follow the reference's."""
    ref = _ref()
    fx = load("ps_small")
    o = _opts(thermostat=thermostat)
    out = Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    _compare(out["thermo"], r["thermo"], 1e-7)
    assert out["thermo"][-1]["volume"] != out["thermo"][0]["volume"]
    np.testing.assert_allclose(out["cell"], r["cell"], rtol=0, atol=1e-9)
    assert np.max(np.abs(out["x"] - r["x"])) < 1e-7


def test_fp64_mtk_temperature_ramp_follows_reference():
    """A ramped target temperature feeds both chains and the volume's mass step by step, as in the reference."""
    ref = _ref()
    fx = load("ps_small")
    o = _opts(temperature=300.0, temperature_end=350.0, steps=20, thermo_every=4)
    out = Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o)
    r = ref.run(fx.ff, fx.x, fx.cell, o)
    _compare(out["thermo"], r["thermo"], 1e-7)


def test_mtk_mixed_runs_and_rejections():
    """The mixed path takes MTK; the reference's refusals hold: constraints, a thermostat other than Nose-Hoover, per-axis
    coupling."""
    fx = load("ps_small")
    o = _opts(precision="mixed", steps=40)
    out = Evaluator(fx.ff, o.energy).run(fx.x, fx.cell, o)
    assert np.all(np.isfinite(out["x"])) and out["thermo"][-1]["volume"] != out["thermo"][0]["volume"]
    for bad, msg in [(dict(constraints="h-bonds"), "without bond constraints"), (dict(thermostat="bussi"), "pairs with the Nos"),
                     (dict(anisotropic=True), "couples the volume isotropically")]:
        b = _opts(**bad)
        with pytest.raises(Exception, match=msg):
            Evaluator(fx.ff, b.energy).run(fx.x, fx.cell, b)
