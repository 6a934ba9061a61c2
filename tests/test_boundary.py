"""The drop-in boundary: the C ABI library exports every entry point include/caps_gpu.h declares, the ctypes mirror
has the C layout, and without a CUDA device the engine refuses loudly (there is no CPU fallback)."""
import ctypes as C
import re
import subprocess
import tempfile
from pathlib import Path

import pytest

from caps_b200 import _abi, build

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "caps_gpu.h"
HEADERS = sorted((ROOT / "include").glob("*.h"))


@pytest.fixture(scope="module")
def lib():
    build.build(verbose=False)
    return _abi.load()


def declared_functions():
    text = "\n".join(h.read_text() for h in HEADERS)
    return sorted(set(re.findall(r"^\s*[A-Za-z_][A-Za-z0-9_ \*]*?\b(caps_gpu_[a-z_]+)\s*\(", text, re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ["caps_gpu_create", "caps_gpu_compute", "caps_gpu_run", "caps_gpu_destroy", "caps_gpu_error"]:
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert set(_abi.EXPORTS) | set(_abi.DIAG_EXPORTS) <= set(declared_functions())
    assert lib.caps_gpu_abi_version() == 5


def test_no_torch_in_the_boundary():
    text = HEADER.read_text()
    assert "torch" not in text.lower() and "at::" not in text


def _c_layout():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "caps_gpu.h"
#define S(T) printf(#T " %zu\n", sizeof(T));
#define O(T, f) printf(#T "." #f " %zu\n", offsetof(T, f));
int main(void) {
  S(caps_gpu_ff) S(caps_gpu_opts) S(caps_gpu_terms) S(caps_gpu_md_opts) S(caps_gpu_thermo) S(caps_gpu_state)
  O(caps_gpu_ff, lj14) O(caps_gpu_ff, excl_offset) O(caps_gpu_ff, model_cutoff) O(caps_gpu_ff, lj_form) O(caps_gpu_ff, fene_k_r0_eps_sigma)
  O(caps_gpu_opts, precision) O(caps_gpu_opts, parts) O(caps_gpu_md_opts, seed) O(caps_gpu_md_opts, is_oxygen) O(caps_gpu_md_opts, checkpoint_every) O(caps_gpu_md_opts, checkpoint_user)
  O(caps_gpu_thermo, p) O(caps_gpu_thermo, terms) O(caps_gpu_terms, tail_virial)
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "l.c"
        c.write_text(src)
        exe = Path(d) / "l"
        subprocess.run(["gcc", "-I", str(ROOT / "include"), str(c), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {k: int(v) for k, v in (line.split() for line in out.strip().splitlines())}


def test_ctypes_layout_matches_c():
    lay = _c_layout()
    py = {"caps_gpu_ff": _abi.FF, "caps_gpu_opts": _abi.Opts, "caps_gpu_terms": _abi.Terms, "caps_gpu_md_opts": _abi.MdOpts,
          "caps_gpu_thermo": _abi.Thermo, "caps_gpu_state": _abi.State}
    for cname, T in py.items():
        assert C.sizeof(T) == lay[cname], cname
    for key, v in lay.items():
        if "." in key:
            cname, f = key.split(".")
            assert getattr(py[cname], f).offset == v, key


def test_without_a_device_the_engine_refuses(lib):
    if lib.caps_gpu_device_count() > 0:
        pytest.skip("a CUDA device is present")
    from caps_b200 import DeviceError, Evaluator
    from tests.fixtures import load
    fx = load("ps_small")
    with pytest.raises(DeviceError, match="no CUDA device"):
        Evaluator(fx.ff, fx.options(0, "mixed"))


def test_library_resolves_all_of_its_own_symbols(lib):
    out = subprocess.run(["nm", "-D", "--undefined-only", str(_abi.LIB_PATH)], capture_output=True, text=True).stdout
    assert "capsb" not in out, [line for line in out.splitlines() if "capsb" in line]
