"""The oracle (oracle/_ref: the reference core built from its sources, with the C++ restatement of its Fortran PME) is
pinned by the reference's own tests and reproduces the committed golden fixtures."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.fixtures import NAMES, load

ROOT = Path(__file__).resolve().parent.parent
REF_SRC = Path("/root/reference/tests")


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built (make -C oracle)")
    return ref


@pytest.mark.skipif(not REF_SRC.exists(), reason="the reference's test sources are not here")
def test_reference_kspace_tests_pass_on_the_restatement():
    """tests/test_kspace.cpp of the reference, unmodified: FFT vs direct DFT, good_size known answers, the Madelung
    constant of rock salt (1.747565), PME vs plain Ewald, threaded half-spectrum PME vs serial PME to 1e-12."""
    _ref()
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "_ref/test_kspace"], check=True, capture_output=True)
    out = subprocess.run([str(ROOT / "oracle" / "_ref" / "test_kspace")], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "4 tests, 0 failed" in out.stdout


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_the_golden_fixture(name):
    ref = _ref()
    fx = load(name)
    for k, _ in fx.cases():
        for prec in ("double", "mixed"):
            t, f = ref.compute(fx.ff, fx.options(k, prec), fx.x, fx.cell, threads=1)
            assert np.array_equal(f, fx.forces[(k, prec)]), (name, k, prec)
            ref_t = fx.terms(k, prec)
            for key in ("bond", "angle", "dihedral", "improper", "vdw", "coulomb", "virial"):
                assert t[key] == ref_t[key], (key, t[key], ref_t[key])


def test_golden_pme_matches_plain_ewald_known_answer():
    """The reference's PME (through the restatement) on the triclinic fixture agrees with the plain Ewald sum, as the
    reference's own test requires (energy 1e-4 relative, forces 1e-3 RMS)."""
    ref = _ref()
    fx = load("lj_triclinic")
    beta = ref.ewald_beta(9.0, 1e-5)
    k = ref.pme_grid(fx.cell, beta, 0.8, 6)
    e, f, vir = ref.pme(fx.x, fx.ff.charge, fx.cell, k, 6, beta)
    assert np.isfinite(e) and np.all(np.isfinite(f))
    assert k == [ref.pme_grid(fx.cell, beta, 0.8, 6)[i] for i in range(3)]
