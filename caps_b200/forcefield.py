"""The force field the device path consumes: the subset of caps::ForceField (core/include/caps/field.hpp:154-249)
that the MD hot path reads, as numpy arrays, and its conversion to the C struct of include/caps_gpu.h.

Also reads the flat binary cell files ("CAPSFF1") written by the oracle's exporter, so cells built by the reference's
own builders can be used here.
"""
from __future__ import annotations

import ctypes as C
import struct
from dataclasses import dataclass, field, fields
from pathlib import Path

import numpy as np

from ._abi import FF


def _u32(a, cols=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint32))
    return a.reshape(-1, cols) if cols else a


def _f64(a, cols=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return a.reshape(-1, cols) if cols else a


@dataclass
class ForceField:
    type_index: np.ndarray                 # [n] int32
    charge: np.ndarray                     # [n] e
    mass: np.ndarray                       # [n] g/mol
    pair_eps: np.ndarray                   # [nt, nt] kcal/mol after mixing
    pair_sigma: np.ndarray                 # [nt, nt] Å
    bond_ij: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.uint32))
    bond_k_r0: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))
    angle_ijk: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.uint32))
    angle_kt_theta0: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))
    dihedral_ijkl: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.uint32))
    dihedral_v_delta: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))
    dihedral_n: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    improper_ijkl: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.uint32))
    improper_v_delta: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))
    improper_n: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    pair14_ij: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.uint32))
    pair14_lj: np.ndarray | None = None
    pair14_coul: np.ndarray | None = None
    lj14: float = 0.5
    coul14: float = 1.0 / 1.2
    excl_offset: np.ndarray | None = None  # [n+1] CSR of the excluded partners
    excl_list: np.ndarray | None = None
    fene_ij: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.uint32))
    fene_k_r0_eps_sigma: np.ndarray = field(default_factory=lambda: np.zeros((0, 4)))
    lj_shift: bool = False
    model_cutoff: float = 0.0
    pair_form: str = "lj12-6"        # "lj12-6" | "lj9-6" (class II)
    element: np.ndarray | None = None      # [n] atomic numbers (constraints: hydrogens, rigid waters)
    # ForceField::pair_func (field.hpp:68, 174): {(a, b): (form, a, b, c, rc)} with form "buckingham" (A, rho, C),
    # "morse" (D, alpha, r0) or "rydberg" (A, rho, C), or their codes 1, 2, 3; rc > 0 the pair's own cut-off
    pair_func: dict | None = None
    lj_inner: float = 0.0                  # ForceField::lj_inner: where the lj/gromacs and CHARMM switches start (Å)
    lj_fsw: bool = False                   # ForceField::lj_fsw: CHARMM's force switch on every 12-6 pair
    tables: list | None = None             # ForceField::tables: [(r0, dr, e[], f[])], pair_func form "table" (a = index)

    def __post_init__(self):
        self.type_index = np.ascontiguousarray(np.asarray(self.type_index, dtype=np.int32))
        self.charge = _f64(self.charge)
        self.mass = _f64(self.mass)
        nt = int(round(np.sqrt(np.asarray(self.pair_eps).size)))
        self.pair_eps = _f64(self.pair_eps).reshape(nt, nt)
        self.pair_sigma = _f64(self.pair_sigma).reshape(nt, nt)
        self.bond_ij, self.bond_k_r0 = _u32(self.bond_ij, 2), _f64(self.bond_k_r0, 2)
        self.angle_ijk, self.angle_kt_theta0 = _u32(self.angle_ijk, 3), _f64(self.angle_kt_theta0, 2)
        self.dihedral_ijkl, self.dihedral_v_delta = _u32(self.dihedral_ijkl, 4), _f64(self.dihedral_v_delta, 2)
        self.dihedral_n = np.ascontiguousarray(np.asarray(self.dihedral_n, dtype=np.int32))
        self.improper_ijkl, self.improper_v_delta = _u32(self.improper_ijkl, 4), _f64(self.improper_v_delta, 2)
        self.improper_n = np.ascontiguousarray(np.asarray(self.improper_n, dtype=np.int32))
        self.pair14_ij = _u32(self.pair14_ij, 2)
        if self.pair14_lj is not None and len(self.pair14_lj) == 0:
            self.pair14_lj = None
        if self.pair14_coul is not None and len(self.pair14_coul) == 0:
            self.pair14_coul = None
        if self.pair14_lj is not None:
            self.pair14_lj = _f64(self.pair14_lj)
        if self.pair14_coul is not None:
            self.pair14_coul = _f64(self.pair14_coul)
        n = self.natoms
        if self.excl_offset is None:
            self.excl_offset = np.zeros(n + 1, np.uint32)
            self.excl_list = np.zeros(0, np.uint32)
        self.excl_offset, self.excl_list = _u32(self.excl_offset), _u32(self.excl_list)
        self.fene_ij, self.fene_k_r0_eps_sigma = _u32(self.fene_ij, 2), _f64(self.fene_k_r0_eps_sigma, 4)
        if self.element is not None:
            self.element = np.ascontiguousarray(np.asarray(self.element, dtype=np.int32))

    @property
    def natoms(self) -> int:
        return int(self.type_index.size)

    @property
    def ntypes(self) -> int:
        return int(self.pair_eps.shape[0])

    def to_struct(self) -> tuple[FF, list]:
        """The C struct pointing into this object's arrays (valid while they live; the list holds references)."""
        keep = []

        def ptr(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a)
            keep.append(a)
            return a.ctypes.data_as(C.c_void_p)

        s = FF()
        s.natoms, s.ntypes = self.natoms, self.ntypes
        s.type_index, s.charge, s.mass = ptr(self.type_index), ptr(self.charge), ptr(self.mass)
        s.pair_eps, s.pair_sigma = ptr(self.pair_eps), ptr(self.pair_sigma)
        s.nbonds, s.bond_ij, s.bond_k_r0 = len(self.bond_ij), ptr(self.bond_ij), ptr(self.bond_k_r0)
        s.nangles, s.angle_ijk, s.angle_kt_theta0 = len(self.angle_ijk), ptr(self.angle_ijk), ptr(self.angle_kt_theta0)
        s.ndihedrals, s.dihedral_ijkl = len(self.dihedral_ijkl), ptr(self.dihedral_ijkl)
        s.dihedral_v_delta, s.dihedral_n = ptr(self.dihedral_v_delta), ptr(self.dihedral_n)
        s.nimpropers, s.improper_ijkl = len(self.improper_ijkl), ptr(self.improper_ijkl)
        s.improper_v_delta, s.improper_n = ptr(self.improper_v_delta), ptr(self.improper_n)
        s.npairs14, s.pair14_ij = len(self.pair14_ij), ptr(self.pair14_ij)
        s.pair14_lj, s.pair14_coul = ptr(self.pair14_lj), ptr(self.pair14_coul)
        s.lj14, s.coul14 = float(self.lj14), float(self.coul14)
        s.excl_offset, s.excl_list = ptr(self.excl_offset), ptr(self.excl_list)
        s.nfene, s.fene_ij, s.fene_k_r0_eps_sigma = len(self.fene_ij), ptr(self.fene_ij), ptr(self.fene_k_r0_eps_sigma)
        s.lj_shift, s.model_cutoff = int(bool(self.lj_shift)), float(self.model_cutoff)
        if self.pair_form not in ("lj12-6", "lj9-6"):
            raise ValueError(f"unknown pair form '{self.pair_form}' (lj12-6, lj9-6)")
        s.lj_form = 1 if self.pair_form == "lj9-6" else 0
        if self.pair_func:
            forms = {"buckingham": 1, "buck": 1, "morse": 2, "rydberg": 3, "sdk9-6": 11, "sdk12-4": 12, "sdk12-6": 13, "sdk12-5": 14,
                     "lj/gromacs": 20, "cos2": 31, "cos2-wca": 32, "table": 40}
            ab, par = [], []
            for (a, b), spec in sorted(self.pair_func.items(), key=lambda kv: (min(kv[0]), max(kv[0]))):
                form, pa, pb, pc = spec[:4]
                rc = spec[4] if len(spec) > 4 else 0.0
                code = forms.get(form.lower()) if isinstance(form, str) else int(form)
                if code is None:
                    raise ValueError(f"unknown pair form {form!r} for types ({a}, {b}) ({', '.join(forms)})")
                ab += [min(a, b), max(a, b)]
                par += [float(code), float(pa), float(pb), float(pc), float(rc)]
            s.npair_func = len(self.pair_func)
            s.pair_func_ab = ptr(np.asarray(ab, dtype=np.int32))
            s.pair_func_p = ptr(np.asarray(par, dtype=np.float64))
        s.lj_inner = float(self.lj_inner)
        s.lj_fsw = int(bool(self.lj_fsw))
        if self.tables:
            s.ntables = len(self.tables)
            s.table_n = ptr(np.asarray([len(t[2]) for t in self.tables], dtype=np.int32))
            s.table_r0_dr = ptr(np.asarray([[float(t[0]), float(t[1])] for t in self.tables], dtype=np.float64))
            s.table_e = ptr(np.concatenate([np.asarray(t[2], dtype=np.float64) for t in self.tables]))
            s.table_f = ptr(np.concatenate([np.asarray(t[3], dtype=np.float64) for t in self.tables]))
        return s, keep

    def arrays(self) -> dict:
        """Every field as a plain dict (for fixtures)."""
        out = {}
        for f in fields(self):
            v = getattr(self, f.name)
            if v is None:
                continue
            out[f.name] = v
        return out

    @classmethod
    def from_arrays(cls, d: dict) -> "ForceField":
        names = {f.name for f in fields(cls)}
        kw = {}
        for k, v in d.items():
            if k not in names:
                continue
            if isinstance(v, np.ndarray) and v.shape == ():
                v = v.item()
            kw[k] = v
        return cls(**kw)


def read_capsff(path: str | Path) -> tuple[ForceField, np.ndarray, np.ndarray, dict]:
    """Reads a CAPSFF1 file: returns (force field, positions [n,3], cell[12], extras)."""
    raw = Path(path).read_bytes()
    if raw[:8] != b"CAPSFF1\n":
        raise ValueError(f"{path}: not a CAPSFF1 file")
    pos, rec = 8, {}
    kinds = {b"d": np.float64, b"i": np.int32, b"u": np.uint32}
    while pos < len(raw):
        head = raw[pos:pos + 40]
        name = head[:32].split(b"\0", 1)[0].decode()
        kind = head[32:33]
        (count,) = struct.unpack("<q", raw[pos + 40:pos + 48])
        pos += 48
        if kind == b"s":
            rec[name] = raw[pos:pos + count].decode(errors="replace")
            pos += count
        else:
            dt = kinds[kind]
            nbytes = count * np.dtype(dt).itemsize
            rec[name] = np.frombuffer(raw[pos:pos + nbytes], dtype=dt).copy()
            pos += nbytes
    n = rec["type_index"].size
    nt = int(round(np.sqrt(rec["pair_eps"].size)))
    lj14, coul14 = rec["lj14_coul14"]
    ff = ForceField(
        type_index=rec["type_index"], charge=rec["charge"], mass=rec["mass"],
        pair_eps=rec["pair_eps"].reshape(nt, nt), pair_sigma=rec["pair_sigma"].reshape(nt, nt),
        bond_ij=rec["bond_ij"], bond_k_r0=rec["bond_k_r0"], angle_ijk=rec["angle_ijk"],
        angle_kt_theta0=rec["angle_kt_theta0"], dihedral_ijkl=rec["dihedral_ijkl"],
        dihedral_v_delta=rec["dihedral_v_delta"], dihedral_n=rec["dihedral_n"], improper_ijkl=rec["improper_ijkl"],
        improper_v_delta=rec["improper_v_delta"], improper_n=rec["improper_n"], pair14_ij=rec["pair14_ij"],
        pair14_lj=rec["pair14_lj"] if rec["pair14_lj"].size else None,
        pair14_coul=rec["pair14_coul"] if rec["pair14_coul"].size else None, lj14=float(lj14), coul14=float(coul14),
        excl_offset=rec["excl_offset"], excl_list=rec["excl_list"], fene_ij=rec["fene_ij"],
        fene_k_r0_eps_sigma=rec["fene_k_r0_eps_sigma"], lj_shift=bool(rec["flags"][0]),
        model_cutoff=float(rec["model_cutoff"][0]), element=rec["element"],
    )
    extras = {"unsupported": int(rec["unsupported"][0]), "name": rec.get("name", ""), "keep13": int(rec["flags"][1])}
    return ff, rec["x"].reshape(n, 3).copy(), rec["cell"].copy(), extras
