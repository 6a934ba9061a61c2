"""ctypes mirror of include/caps_gpu.h and the loader of the device library.

The product path is the C ABI in libcaps_b200.so; this module only binds it. There is no CPU fallback: when the library
or a CUDA device is missing, the calls that need them raise.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libcaps_b200.so"

P = C.c_void_p


class FF(C.Structure):
    _fields_ = [
        ("natoms", C.c_int32), ("ntypes", C.c_int32),
        ("type_index", P), ("charge", P), ("mass", P), ("pair_eps", P), ("pair_sigma", P),
        ("nbonds", C.c_int32), ("bond_ij", P), ("bond_k_r0", P),
        ("nangles", C.c_int32), ("angle_ijk", P), ("angle_kt_theta0", P),
        ("ndihedrals", C.c_int32), ("dihedral_ijkl", P), ("dihedral_v_delta", P), ("dihedral_n", P),
        ("nimpropers", C.c_int32), ("improper_ijkl", P), ("improper_v_delta", P), ("improper_n", P),
        ("npairs14", C.c_int32), ("pair14_ij", P), ("pair14_lj", P), ("pair14_coul", P),
        ("lj14", C.c_double), ("coul14", C.c_double),
        ("excl_offset", P), ("excl_list", P),
        ("nfene", C.c_int32), ("fene_ij", P), ("fene_k_r0_eps_sigma", P),
        ("lj_shift", C.c_int32), ("model_cutoff", C.c_double), ("lj_form", C.c_int32),
        # ABI 5
        ("npair_func", C.c_int32), ("pair_func_ab", C.c_void_p), ("pair_func_p", C.c_void_p),
        ("lj_inner", C.c_double), ("lj_fsw", C.c_int32), ("ntables", C.c_int32), ("table_n", C.c_void_p), ("table_r0_dr", C.c_void_p),
        ("table_e", C.c_void_p), ("table_f", C.c_void_p),
    ]


class Opts(C.Structure):
    _fields_ = [
        ("cutoff", C.c_double), ("skin", C.c_double), ("coulomb", C.c_int32), ("electrostatics", C.c_int32),
        ("dsf_alpha", C.c_double), ("ewald_rtol", C.c_double), ("pme_spacing", C.c_double), ("pme_order", C.c_int32),
        ("tail", C.c_int32), ("precision", C.c_int32), ("force_cap", C.c_double), ("parts", C.c_int32),
    ]


class Terms(C.Structure):
    _fields_ = [
        ("bond", C.c_double), ("angle", C.c_double), ("dihedral", C.c_double), ("improper", C.c_double),
        ("vdw", C.c_double), ("coulomb", C.c_double), ("virial", C.c_double), ("w", C.c_double * 6),
        ("tail_energy", C.c_double), ("tail_virial", C.c_double),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "w"}
        d["w"] = [self.w[i] for i in range(6)]
        d["total"] = self.bond + self.angle + self.dihedral + self.improper + self.vdw + self.coulomb
        return d


class MdOpts(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("steps", C.c_int64), ("temperature", C.c_double), ("temperature_end", C.c_double),
        ("thermostat", C.c_int32), ("tau_t", C.c_double), ("barostat", C.c_int32), ("pressure", C.c_double),
        ("tau_p", C.c_double), ("compressibility", C.c_double), ("barostat_every", C.c_int32),
        ("constraints", C.c_int32), ("new_velocities", C.c_int32), ("seed", C.c_uint64), ("thermo_every", C.c_int32),
        ("frame_every", C.c_int32), ("step_offset", C.c_int64), ("respa", C.c_int32),
        ("is_hydrogen", P), ("is_oxygen", P), ("respa_split", C.c_int32),
        ("checkpoint_every", C.c_int64), ("checkpoint", C.c_void_p), ("checkpoint_user", C.c_void_p),
        ("hmr", C.c_double), ("anisotropic", C.c_int32), ("couple_axes", C.c_int32), ("axis_pressure_set", C.c_int32),
        ("axis_pressure", C.c_double * 3),
        # ABI 5
        ("constraint_algorithm", C.c_int32),
    ]


class Thermo(C.Structure):
    _fields_ = [
        ("step", C.c_int64), ("time_ps", C.c_double), ("temperature", C.c_double), ("potential", C.c_double),
        ("kinetic", C.c_double), ("total", C.c_double), ("conserved", C.c_double), ("pressure", C.c_double),
        ("volume", C.c_double), ("density", C.c_double), ("target_temperature", C.c_double), ("p", C.c_double * 6),
        ("terms", Terms),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("p", "terms")}
        d["p"] = [self.p[i] for i in range(6)]
        d["terms"] = self.terms.as_dict()
        return d


class State(C.Structure):
    _fields_ = [("x", P), ("v", P), ("cell", P), ("has_velocities", C.c_int32)]


PROGRESS_FN = C.CFUNCTYPE(C.c_int32, C.POINTER(Thermo), C.c_void_p)
FRAME_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64, C.c_void_p)
CHECKPOINT_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64, C.c_void_p)

DIAG_EXPORTS = ["caps_gpu_diag_set_timing", "caps_gpu_diag_last_step_ms", "caps_gpu_diag_pair_timing", "caps_gpu_diag_step_kernels",
                "caps_gpu_diag_kernels_run", "caps_gpu_diag_list_counts", "caps_gpu_diag_phase_timing", "caps_gpu_diag_get_tuning", "caps_gpu_diag_set_tuning"]

EXPORTS = [
    "caps_gpu_abi_version", "caps_gpu_device_count", "caps_gpu_create", "caps_gpu_set_options", "caps_gpu_energies",
    "caps_gpu_compute", "caps_gpu_compute_device", "caps_gpu_list_builds", "caps_gpu_run", "caps_gpu_run_batch",
    "caps_gpu_last_steps_per_second", "caps_gpu_destroy", "caps_gpu_error",
    "caps_gpu_request_stop", "caps_gpu_stop_requested", "caps_gpu_traj_open", "caps_gpu_traj_append", "caps_gpu_traj_frame",
    "caps_gpu_traj_frames", "caps_gpu_traj_close", "caps_gpu_reload", "caps_gpu_freeze_pairs", "caps_gpu_unfreeze", "caps_gpu_pairs",
    "caps_gpu_threads",
]

_lib = None


def load(path: Path | None = None) -> C.CDLL:
    """The device library, with its signatures declared. Raises when it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m caps_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(str(p))
    lib.caps_gpu_abi_version.restype = C.c_int32
    lib.caps_gpu_device_count.restype = C.c_int32
    lib.caps_gpu_create.restype = C.c_void_p
    lib.caps_gpu_create.argtypes = [C.POINTER(FF), C.POINTER(Opts)]
    lib.caps_gpu_set_options.argtypes = [C.c_void_p, C.POINTER(Opts)]
    lib.caps_gpu_energies.argtypes = [C.c_void_p, C.c_int32]
    lib.caps_gpu_compute.argtypes = [C.c_void_p, P, P, P, C.POINTER(Terms)]
    lib.caps_gpu_compute_device.argtypes = [C.c_void_p, P, P, P, C.POINTER(Terms)]
    lib.caps_gpu_list_builds.argtypes = [C.c_void_p]
    lib.caps_gpu_run.argtypes = [C.c_void_p, C.POINTER(State), C.POINTER(MdOpts), PROGRESS_FN, FRAME_FN, C.c_void_p,
                                 C.c_char_p, C.c_int32]
    lib.caps_gpu_last_steps_per_second.restype = C.c_double
    lib.caps_gpu_last_steps_per_second.argtypes = [C.c_void_p]
    lib.caps_gpu_run_batch.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int32, PROGRESS_FN, FRAME_FN,
                                       C.POINTER(C.c_void_p)]
    lib.caps_gpu_destroy.argtypes = [C.c_void_p]
    lib.caps_gpu_error.restype = C.c_char_p
    lib.caps_gpu_error.argtypes = [C.c_void_p]
    lib.caps_gpu_reload.argtypes = [C.c_void_p, C.POINTER(FF)]
    lib.caps_gpu_freeze_pairs.argtypes = [C.c_void_p, P, P]
    lib.caps_gpu_unfreeze.argtypes = [C.c_void_p]
    lib.caps_gpu_pairs.restype = C.c_int64
    lib.caps_gpu_pairs.argtypes = [C.c_void_p]
    lib.caps_gpu_threads.argtypes = [C.c_void_p]
    lib.caps_gpu_request_stop.argtypes = [C.c_int32]
    lib.caps_gpu_stop_requested.restype = C.c_int32
    lib.caps_gpu_traj_open.restype = C.c_void_p
    lib.caps_gpu_traj_open.argtypes = [C.c_char_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_double]
    lib.caps_gpu_traj_append.argtypes = [C.c_void_p, P, P, C.c_int64]
    lib.caps_gpu_traj_frame.argtypes = [P, P, C.c_int64, C.c_void_p]
    lib.caps_gpu_traj_frames.restype = C.c_int64
    lib.caps_gpu_traj_frames.argtypes = [C.c_void_p]
    lib.caps_gpu_traj_close.argtypes = [C.c_void_p]
    # measurement entry points (include/caps_gpu_diag.h)
    lib.caps_gpu_diag_set_timing.argtypes = [C.c_void_p, C.c_int64]
    lib.caps_gpu_diag_last_step_ms.restype = C.c_double
    lib.caps_gpu_diag_last_step_ms.argtypes = [C.c_void_p]
    lib.caps_gpu_diag_step_kernels.argtypes = [C.c_void_p]
    lib.caps_gpu_diag_kernels_run.restype = C.c_int64
    lib.caps_gpu_diag_kernels_run.argtypes = [C.c_void_p]
    lib.caps_gpu_diag_list_counts.restype = C.c_int32
    lib.caps_gpu_diag_list_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    lib.caps_gpu_diag_pair_timing.argtypes = [C.c_void_p, P, P, C.c_int32, C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                              C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.caps_gpu_diag_phase_timing.argtypes = [C.c_void_p, P, P, C.c_int32, C.c_int64, P]
    lib.caps_gpu_diag_get_tuning.argtypes = [C.c_void_p, P]
    lib.caps_gpu_diag_set_tuning.argtypes = [C.c_void_p, P]
    if path is None:
        _lib = lib
    return lib
