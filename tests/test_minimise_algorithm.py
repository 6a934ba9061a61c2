"""The minimiser's iteration (caps_b200.minimise: directions, backtracking line search, L-BFGS history, FIRE) against
the reference's minimise (core/src/relax.cpp:65), both driven by the reference's own FP64 forces: with the same forces
the same method must take the same path, so the energies after a fixed number of iterations agree to rounding. Needs no
GPU (the evaluator here is the reference core)."""
import numpy as np
import pytest

from caps_b200 import EnergyOptions
from caps_b200.minimise import MinimiseOptions, minimise
from tests.fixtures import load


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


class RefEvaluator:
    """compute() through the reference core (FP64), in the Evaluator's calling convention."""

    def __init__(self, ref, ff, opts):
        self.ref, self.ff, self.opts = ref, ff, opts

    def compute(self, x, cell):
        return self.ref.compute(self.ff, self.opts, x, cell)


@pytest.mark.parametrize("method", ["sd", "cg", "lbfgs", "fire"])
def test_minimise_path_matches_reference(method):
    ref = _ref()
    fx = load("lj_triclinic")
    eo = EnergyOptions(cutoff=8.0, skin=2.0, electrostatics="dsf", precision="double")
    n = fx.x.shape[0]
    fixed = np.zeros(n, dtype=np.int8)
    fixed[:3] = 1          # held atoms
    fixed[3] = 2 | 8       # x and z of one atom held
    mo = MinimiseOptions(method=method, ftol=1e-6, etol=0.0, max_iterations=25, fixed=list(fixed),
                         restraints=[(5, 9, 3.0, 20.0)], dihedral_restraints=[(10, 11, 12, 13, 60.0, 5.0)])
    mine = minimise(RefEvaluator(ref, fx.ff, eo), fx.x, fx.cell, mo)
    theirs = ref.minimise(fx.ff, eo, fx.x, fx.cell, mo)
    assert mine["stopped_by"] == theirs["stopped_by"]
    assert mine["iterations"] == theirs["iterations"] and mine["evaluations"] == theirs["evaluations"]
    assert abs(mine["energy"] - theirs["energy"]) <= 1e-9 * max(1.0, abs(theirs["energy"]))
    assert np.max(np.abs(mine["x"] - theirs["x"])) < 1e-7
    assert np.array_equal(mine["x"][:3], np.asarray(fx.x)[:3])


def test_minimise_rejects_unknown_method():
    with pytest.raises(ValueError):
        minimise(None, np.zeros((1, 3)), np.zeros(12), MinimiseOptions(method="newton"))
