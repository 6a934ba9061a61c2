"""The allocation-free entry point, caps_gpu_kinetic_noalloc (include/caps_gpu.h).

It serves callers that may not call cudaMalloc (a host whose memory manager owns all device memory, or code beside a
long stream-ordered pipeline that an allocation would synchronise): they pass their own device buffers, and the only
working memory is a fixed array inside the library. Its kinetic energy and kinetic tensor must equal what the run entry
point (caps_gpu_run) reports for the same velocities in its step-0 thermo row, and what plain FP64 sums in numpy give
for the same velocities and masses. Two calls in a row, the second on fewer
atoms than the first, check that the shared working memory carries nothing from one call to the next.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from caps_b200 import DynamicsOptions, Evaluator, _abi
from tests.fixtures import load

pytestmark = pytest.mark.gpu

K_ATM = 68568.415   # kcal/(mol Å^3) -> atm, as the run's thermo rows use
K_ACC = 4.184e-4    # (kcal/mol/Å)/(g/mol) -> Å/fs², the unit factor of the kinetic energy
TOL = 1e-12         # the FP64 tolerance of the device parity tests


def _reference_row(fx, v):
    """Step-0 thermo row of caps_gpu_run with velocities v (no thermostat, no constraints, no steps)."""
    o = DynamicsOptions(dt=1.0, steps=0, temperature=300.0, thermostat="none", thermo_every=1, seed=3,
                        energy=fx.options(0, "double"))
    ev = Evaluator(fx.ff, o.energy)
    out = ev.run(fx.x, fx.cell, o, v=v)
    ev.close()
    return out["thermo"][0]


def _noalloc(lib, v, mass):
    torch = pytest.importorskip("torch")
    dv = torch.tensor(np.ascontiguousarray(v, dtype=np.float64).reshape(-1), device="cuda")
    dm = torch.tensor(np.ascontiguousarray(mass, dtype=np.float64), device="cuda")
    out = torch.full((7,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.caps_gpu_kinetic_noalloc(C.c_void_p(dv.data_ptr()), C.c_void_p(dm.data_ptr()), C.c_int32(len(mass)),
                                      C.c_void_p(out.data_ptr()), C.c_void_p(0))
    assert rc == 0, lib.caps_gpu_error(None).decode()
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.fixture(scope="module")
def lib():
    lib = _abi.load()
    lib.caps_gpu_kinetic_noalloc.restype = C.c_int32
    lib.caps_gpu_kinetic_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
    return lib


def test_noalloc_kinetic_matches_run_twice(lib):
    rng = np.random.default_rng(11)
    results = []
    for name in ("lj_triclinic", "kg"):   # 1100 atoms, then 500: the second call reads fewer partial sums
        fx = load(name)
        n = fx.ff.natoms
        v = rng.normal(0.0, 0.01, size=(n, 3))
        row = _reference_row(fx, v)
        got = _noalloc(lib, v, fx.ff.mass)
        ke = row["kinetic"]
        assert abs(got[0] - ke) <= TOL * abs(ke), (name, got[0], ke)
        # the kinetic tensor behind the row's pressure tensor: p_c V / kAtm - W_c
        kin = np.array([row["p"][c] * row["volume"] / K_ATM - row["terms"]["w"][c] for c in range(6)])
        scale = max(abs(ke), max(abs(w) for w in row["terms"]["w"]))
        assert np.max(np.abs(got[1:] - kin)) <= 1e-10 * scale, (name, got[1:], kin)
        assert abs(got[1] + got[2] + got[3] - 2 * got[0]) <= TOL * abs(ke)
        # and against plain FP64 sums in numpy, independent of the engine: 0.5 sum m v^2 and sum m v_a v_b, in kcal/mol
        m = np.asarray(fx.ff.mass, dtype=np.float64)
        ke_np = 0.5 * np.sum(m[:, None] * v * v) / K_ACC
        pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
        kin_np = np.array([np.sum(m * v[:, a] * v[:, b]) for a, b in pairs]) / K_ACC
        assert abs(got[0] - ke_np) <= TOL * abs(ke_np), (name, got[0], ke_np)
        assert np.max(np.abs(got[1:] - kin_np)) <= TOL * abs(ke_np), (name, got[1:], kin_np)
        results.append(got)
    assert results[0][0] != results[1][0]


def test_noalloc_rejects_sizes_beyond_its_memory(lib):
    torch = pytest.importorskip("torch")
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    assert lib.caps_gpu_kinetic_noalloc(p, p, C.c_int32((1 << 20) + 1), p, None) == -1
    assert b"outside" in lib.caps_gpu_error(None)
    assert lib.caps_gpu_kinetic_noalloc(p, p, C.c_int32(0), p, None) == -1
