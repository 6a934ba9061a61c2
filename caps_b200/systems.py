"""Synthetic cells of the benchmark shapes, built from seeds (no files, no network).

polystyrene_melt: atactic polystyrene, 16 atoms per repeat unit, OPLS-AA-style parameters (geometric mixing, 1-4 at 0.5,
aromatic C -0.115 / H +0.115, backbone CH2 and CH balanced to neutral), grown as random-walk chains in a cubic box at
the target density. kg_melt: Kremer-Grest bead-spring chains (WCA + FENE). spce_water: rigid SPC/E water on a jittered
lattice with random orientations. The geometry code is this package's own; the overlaps a dense growth leaves are
removed by push_off (capped-force FP64 MD on the device) before a run.
"""
from __future__ import annotations

import math

import numpy as np

from .forcefield import ForceField

KB = 0.0019872041   # kcal/(mol K)
NA = 6.02214076e23
M_C, M_H, M_O = 12.011, 1.008, 15.999


# --- topology helpers -----------------------------------------------------------------------------------------
def _graph(n: int, bonds: np.ndarray) -> list[list[int]]:
    nb = [[] for _ in range(n)]
    for i, j in bonds:
        nb[int(i)].append(int(j))
        nb[int(j)].append(int(i))
    return nb


def angles_from_bonds(nb: list[list[int]]) -> np.ndarray:
    out = []
    for j, ns in enumerate(nb):
        for a in range(len(ns)):
            for b in range(a + 1, len(ns)):
                out.append((ns[a], j, ns[b]))
    return np.array(out, dtype=np.uint32).reshape(-1, 3)


def dihedrals_from_bonds(nb: list[list[int]], bonds: np.ndarray) -> np.ndarray:
    out = []
    for j, k in bonds:
        j, k = int(j), int(k)
        for i in nb[j]:
            if i == k:
                continue
            for l in nb[k]:
                if l == j or l == i:
                    continue
                out.append((i, j, k, l))
    return np.array(out, dtype=np.uint32).reshape(-1, 4)


def exclusions(n: int, nb: list[list[int]], depth: int = 3) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """CSR of partners within `depth` bonds, and the 1-4 pairs (exactly 3 bonds apart, not closer)."""
    off = np.zeros(n + 1, np.uint32)
    lst, p14 = [], []
    for i in range(n):
        dist = {i: 0}
        frontier = [i]
        for d in range(1, depth + 1):
            nxt = []
            for a in frontier:
                for b in nb[a]:
                    if b not in dist:
                        dist[b] = d
                        nxt.append(b)
            frontier = nxt
        part = sorted(j for j in dist if j != i)
        lst += part
        off[i + 1] = len(lst)
        p14 += [(i, j) for j in part if dist[j] == 3 and j > i]
    return off, np.array(lst, np.uint32), np.array(p14, np.uint32).reshape(-1, 2)


def _unit(v):
    return v / np.linalg.norm(v)


def _nerf(a, b, c, bond, angle, torsion):
    """Position of d with |cd| = bond, angle bcd, dihedral abcd (radians)."""
    bc = _unit(c - b)
    nrm = _unit(np.cross(b - a, bc))
    m = np.array([bc, np.cross(nrm, bc), nrm]).T
    d2 = np.array([-bond * math.cos(angle), bond * math.sin(angle) * math.cos(torsion), bond * math.sin(angle) * math.sin(torsion)])
    return c + m @ d2


class _Grid:
    """A cell list over a periodic cubic box for overlap checks while growing."""

    def __init__(self, L: float, cell: float = 3.2, cap: int = 24):
        self.L = L
        self.n = max(3, int(L / cell))
        self.h = L / self.n
        self.cap = cap
        self.cnt = np.zeros((self.n,) * 3, np.int32)
        self.idx = np.full((self.n,) * 3 + (cap,), -1, np.int64)
        self.pos: list[np.ndarray] = []

    def add(self, p: np.ndarray, owner: int):
        c = tuple((np.floor(p / self.h).astype(int)) % self.n)
        k = self.cnt[c]
        if k < self.cap:
            self.idx[c + (k,)] = len(self.pos)
            self.cnt[c] += 1
        self.pos.append(np.asarray(p, float))

    def min_dist(self, pts: np.ndarray, skip_from: int) -> float:
        """Smallest distance from pts to stored atoms with index < skip_from (minimum image)."""
        if not self.pos or skip_from <= 0:
            return 1e9
        P = np.array(self.pos[:skip_from]) if False else None  # noqa: F841  (kept lazy below)
        cells = np.floor(pts / self.h).astype(int)
        lo, hi = cells.min(0) - 1, cells.max(0) + 2
        ids = []
        for a in range(lo[0], hi[0]):
            for b in range(lo[1], hi[1]):
                for c in range(lo[2], hi[2]):
                    t = (a % self.n, b % self.n, c % self.n)
                    k = self.cnt[t]
                    if k:
                        ids.append(self.idx[t][:k])
        if not ids:
            return 1e9
        ids = np.concatenate(ids)
        ids = ids[ids < skip_from]
        if ids.size == 0:
            return 1e9
        Q = np.array([self.pos[i] for i in ids])
        d = pts[:, None, :] - Q[None, :, :]
        d -= self.L * np.round(d / self.L)
        return float(np.sqrt((d * d).sum(-1)).min())


# OPLS-AA-style parameters (kcal/mol, Å, degrees): classes CT (sp3 C), CA (aromatic C), HC, HA
_LJ = {"CT": (0.066, 3.50), "CA": (0.070, 3.55), "HC": (0.030, 2.50), "HA": (0.030, 2.42)}
_BOND = {("CT", "CT"): (268.0, 1.529), ("CT", "HC"): (340.0, 1.090), ("CA", "CA"): (469.0, 1.400), ("CA", "HA"): (367.0, 1.080),
         ("CA", "CT"): (317.0, 1.510)}
_ANGLE = {("CT", "CT", "CT"): (58.35, 112.7), ("CT", "CT", "HC"): (37.5, 110.7), ("HC", "CT", "HC"): (33.0, 107.8),
          ("CA", "CT", "CT"): (63.0, 114.0), ("CA", "CT", "HC"): (35.0, 109.5), ("CA", "CA", "CT"): (70.0, 120.0),
          ("CA", "CA", "CA"): (63.0, 120.0), ("CA", "CA", "HA"): (35.0, 120.0)}
# OPLS Fourier V1, V2, V3 (E = V1/2 (1 + cos phi) + V2/2 (1 - cos 2 phi) + V3/2 (1 + cos 3 phi))
_TORS = {("CT", "CT", "CT", "CT"): (1.740, -0.157, 0.279), ("CT", "CT", "CT", "HC"): (0.0, 0.0, 0.300),
         ("HC", "CT", "CT", "HC"): (0.0, 0.0, 0.300), ("CA", "CA", "CA", "CA"): (0.0, 7.250, 0.0),
         ("CA", "CA", "CA", "HA"): (0.0, 7.250, 0.0), ("HA", "CA", "CA", "HA"): (0.0, 7.250, 0.0),
         ("CA", "CA", "CA", "CT"): (0.0, 7.250, 0.0), ("CT", "CA", "CA", "HA"): (0.0, 7.250, 0.0),
         ("CA", "CA", "CT", "CT"): (0.0, 0.0, 0.0), ("CA", "CA", "CT", "HC"): (0.0, 0.0, 0.0),
         ("CA", "CT", "CT", "CT"): (-2.4, 0.0, 0.0), ("CA", "CT", "CT", "HC"): (0.0, 0.0, 0.462),
         ("CA", "CT", "CT", "CA"): (0.0, 0.0, 0.0)}
_Q = {"CA": -0.115, "HA": 0.115}


def _key_sym(d: dict, k: tuple):
    if k in d:
        return d[k]
    return d.get(tuple(reversed(k)))


def polystyrene_melt(chains: int = 40, dp: int = 50, density: float = 1.04, seed: int = 1, min_sep: float = 2.4,
                     trials: int = 24, grow: bool = True) -> tuple[ForceField, np.ndarray, np.ndarray]:
    """Atactic polystyrene, `chains` x `dp` repeat units of 16 atoms (CH2-CH(C6H5), chain ends left open so the count
    is exactly 16 per unit), at `density` g/cm^3 in a cubic periodic box. Returns (force field, x [n,3], cell[12]).
    grow=False skips the geometry (positions left zero; the topology and force field do not depend on it)."""
    rng = np.random.default_rng(seed)
    n_unit = 16
    n = chains * dp * n_unit
    mass_unit = 8 * M_C + 8 * M_H
    L = (chains * dp * mass_unit / (density * NA) * 1e24) ** (1.0 / 3.0)
    grid = _Grid(L)
    x = np.zeros((n, 3))
    cls = [""] * n
    bonds = []
    tet = math.radians(112.7)
    for ch in range(chains):
        base = ch * dp * n_unit
        # backbone: CH2 (index 0 of a unit) and CH (index 1); three seed points for the NeRF frames
        p0 = rng.uniform(0, L, 3)
        d1 = _unit(rng.normal(size=3))
        p1 = p0 + 1.529 * d1
        perp = _unit(np.cross(d1, _unit(rng.normal(size=3))))
        p_prev2 = p0 - 1.529 * (math.cos(math.pi - tet) * d1 + math.sin(math.pi - tet) * perp)
        bb = [p_prev2, p0, p1]
        chain_first_atom = len(grid.pos)
        for u in range(dp):
            a_ch2, a_ch = base + u * n_unit, base + u * n_unit + 1
            best, best_d = None, -1.0
            for _ in range(trials if grow else 1):
                if u == 0:
                    q_ch2, q_ch = bb[1], bb[2]
                    q_prev = bb[0]
                else:
                    t1 = rng.choice([math.pi, math.pi / 3, -math.pi / 3], p=[0.6, 0.2, 0.2])
                    t2 = rng.choice([math.pi, math.pi / 3, -math.pi / 3], p=[0.6, 0.2, 0.2])
                    q_ch2 = _nerf(bb[-3], bb[-2], bb[-1], 1.529, tet, t1)
                    q_ch = _nerf(bb[-2], bb[-1], q_ch2, 1.529, tet, t2)
                    q_prev = bb[-1]
                # the next backbone atom direction (for the CH's tetrahedral sites)
                q_next = _nerf(q_prev, q_ch2, q_ch, 1.529, tet, math.pi)
                u1, u2 = _unit(q_ch2 - q_ch), _unit(q_next - q_ch)
                bis, nrm = _unit(-(u1 + u2)), _unit(np.cross(u1, u2))
                side = 1.0 if rng.random() < 0.5 else -1.0     # tacticity: which site holds the ring
                ang = math.radians(54.75)
                d_ring = _unit(bis * math.cos(ang) + side * nrm * math.sin(ang))
                d_h = _unit(bis * math.cos(ang) - side * nrm * math.sin(ang))
                ipso = q_ch + 1.510 * d_ring
                centre = ipso + 1.400 * d_ring
                e2 = _unit(np.cross(d_ring, _unit(rng.normal(size=3))))
                e3 = np.cross(d_ring, e2)
                ring = [centre + 1.400 * (-d_ring * math.cos(math.radians(60 * k)) + e2 * math.sin(math.radians(60 * k))) for k in range(6)]
                ring_h = [centre + 2.480 * _unit(r - centre) for r in ring[1:]]
                # CH2 hydrogens: the two sites of a tetrahedral carbon between q_prev and q_ch
                v1, v2 = _unit(q_prev - q_ch2), _unit(q_ch - q_ch2)
                b2, n2 = _unit(-(v1 + v2)), _unit(np.cross(v1, v2))
                h2a = q_ch2 + 1.090 * _unit(b2 * math.cos(ang) + n2 * math.sin(ang))
                h2b = q_ch2 + 1.090 * _unit(b2 * math.cos(ang) - n2 * math.sin(ang))
                h1 = q_ch + 1.090 * d_h
                pts = np.array([q_ch2, q_ch, h2a, h2b, h1] + ring + ring_h)
                del e3
                dmin = grid.min_dist(np.mod(pts, L), max(chain_first_atom, len(grid.pos) - 2 * n_unit)) if grow else 1e9
                if dmin > best_d:
                    best, best_d = pts, dmin
                if dmin >= min_sep:
                    break
            pts = best
            bb.extend([pts[0], pts[1]]) if u > 0 else None
            if u == 0:
                bb = [bb[0], pts[0], pts[1]]
            # atom order in the unit: CH2 C, CH C, 2 H on CH2, H on CH, ring C ipso..C6, ring H 2..6
            order = [0, 1, 2, 3, 4] + list(range(5, 11)) + list(range(11, 16))
            for k, idx in enumerate(order):
                x[base + u * n_unit + k] = pts[idx]
                if grow:
                    grid.add(np.mod(pts[idx], L), base + u * n_unit + k)
            o = base + u * n_unit
            cls[o:o + 16] = ["CT", "CT", "HC", "HC", "HC"] + ["CA"] * 6 + ["HA"] * 5
            bonds += [(o, o + 1), (o, o + 2), (o, o + 3), (o + 1, o + 4), (o + 1, o + 5)]
            for k in range(6):
                bonds.append((o + 5 + k, o + 5 + (k + 1) % 6))
            for k in range(5):
                bonds.append((o + 6 + k, o + 11 + k))
            if u > 0:
                bonds.append((o - n_unit + 1, o))   # CH of the previous unit to this CH2
    bonds = np.array(bonds, np.uint32)
    nb = _graph(n, bonds)
    types = ["CT", "CA", "HC", "HA"]
    tidx = np.array([types.index(c) for c in cls], np.int32)
    eps = np.array([_LJ[t][0] for t in types])
    sig = np.array([_LJ[t][1] for t in types])
    q = np.array([_Q.get(c, 0.0) for c in cls])
    # backbone balanced to neutral per unit: the ipso carbon carries nothing, the 6 aromatic CH pairs are neutral;
    # the ring's C-H pairs (5) sum to 0, so the backbone stays at 0: CH2 C -0.12, its H +0.06 each; CH C -0.06, H +0.06
    for u0 in range(0, n, n_unit):
        q[u0 + 5] = 0.0          # ipso carbon
        q[u0] = -0.12
        q[u0 + 2] = q[u0 + 3] = 0.06
        q[u0 + 1] = -0.06
        q[u0 + 4] = 0.06
    mass = np.array([M_C if c in ("CT", "CA") else M_H for c in cls])
    bk = np.array([_key_sym(_BOND, (cls[i], cls[j])) for i, j in bonds])
    ang = angles_from_bonds(nb)
    ak = []
    for i, j, k in ang:
        kt, th = _key_sym(_ANGLE, (cls[i], cls[j], cls[k]))
        ak.append((kt, math.radians(th)))
    dih = dihedrals_from_bonds(nb, bonds)
    d_ijkl, d_vd, d_n = [], [], []
    for i, j, k, l in dih:
        v = _key_sym(_TORS, (cls[i], cls[j], cls[k], cls[l]))
        if v is None:
            continue
        for nn, (vv, delta) in enumerate(((v[0] / 2, 0.0), (v[1] / 2, math.pi), (v[2] / 2, 0.0)), start=1):
            if vv != 0.0:
                d_ijkl.append((i, j, k, l))
                d_vd.append((vv, delta))
                d_n.append(nn)
    # impropers keeping the ring and its substituents planar: v [1 + cos(2 phi - pi)], v = 1.1 (OPLS aromatic)
    imp_ijkl, imp_vd, imp_n = [], [], []
    for u0 in range(0, n, n_unit):
        for k in range(6):
            c = u0 + 5 + k
            sub = u0 + 1 if k == 0 else u0 + 11 + (k - 1)
            a, b = u0 + 5 + (k - 1) % 6, u0 + 5 + (k + 1) % 6
            imp_ijkl.append((a, b, c, sub))
            imp_vd.append((1.1, math.pi))
            imp_n.append(2)
    off, lst, p14 = exclusions(n, nb)
    pe = np.sqrt(np.outer(eps, eps))
    ps = np.sqrt(np.outer(sig, sig))
    el = np.array([6 if c in ("CT", "CA") else 1 for c in cls], np.int32)
    ff = ForceField(type_index=tidx, charge=q, mass=mass, pair_eps=pe, pair_sigma=ps, bond_ij=bonds, bond_k_r0=bk,
                    angle_ijk=ang, angle_kt_theta0=np.array(ak), dihedral_ijkl=np.array(d_ijkl, np.uint32).reshape(-1, 4),
                    dihedral_v_delta=np.array(d_vd).reshape(-1, 2), dihedral_n=np.array(d_n, np.int32),
                    improper_ijkl=np.array(imp_ijkl, np.uint32), improper_v_delta=np.array(imp_vd), improper_n=np.array(imp_n, np.int32),
                    pair14_ij=p14, lj14=0.5, coul14=0.5, excl_offset=off, excl_list=lst, element=el)
    cell = np.array([0, 0, 0, L, 0, 0, 0, L, 0, 0, 0, L], float)
    return ff, x, cell


def kg_melt(chains: int = 100, beads: int = 50, density: float = 0.85, seed: int = 1, bond: float = 0.97):
    """Kremer-Grest chains in reduced units mapped as sigma = 1 Å, eps = 1 kcal/mol, m = 1 g/mol: WCA (cut-off
    2^(1/6), shifted), FENE K = 30, R0 = 1.5 with the WCA core on bonded pairs, 1-2 pairs excluded from the WCA pairs."""
    rng = np.random.default_rng(seed)
    n = chains * beads
    L = (n / density) ** (1.0 / 3.0)
    x = np.zeros((n, 3))
    for c in range(chains):
        p = rng.uniform(0, L, 3)
        prev = None
        for k in range(beads):
            if k:
                for _ in range(1000):
                    d = _unit(rng.normal(size=3))
                    if prev is None or np.dot(d, prev) > -0.5:
                        break
                p = p + bond * d
                prev = d
            x[c * beads + k] = p
    bonds = np.array([(c * beads + k, c * beads + k + 1) for c in range(chains) for k in range(beads - 1)], np.uint32)
    nb = _graph(n, bonds)
    off, lst, _ = exclusions(n, nb, depth=1)
    ff = ForceField(type_index=np.zeros(n, np.int32), charge=np.zeros(n), mass=np.ones(n), pair_eps=[[1.0]], pair_sigma=[[1.0]],
                    fene_ij=bonds, fene_k_r0_eps_sigma=np.tile([30.0, 1.5, 1.0, 1.0], (len(bonds), 1)), excl_offset=off,
                    excl_list=lst, lj_shift=True, model_cutoff=2 ** (1 / 6), element=np.zeros(n, np.int32))
    cell = np.array([0, 0, 0, L, 0, 0, 0, L, 0, 0, 0, L], float)
    return ff, x, cell


def spce_water(nmol: int = 100000, density: float = 0.997, seed: int = 1):
    """Rigid SPC/E water (O-H 1.0 Å, H-O-H 109.47 degrees; O sigma 3.166 Å, eps 0.650 kJ/mol; q_O -0.8476, q_H
    +0.4238) on a jittered cubic lattice with random orientations."""
    rng = np.random.default_rng(seed)
    mass_mol = M_O + 2 * M_H
    L = (nmol * mass_mol / (density * NA) * 1e24) ** (1.0 / 3.0)
    m = int(math.ceil(nmol ** (1.0 / 3.0)))
    a = L / m
    sites = np.array([(i, j, k) for i in range(m) for j in range(m) for k in range(m)], float)[:nmol]
    o = (sites + 0.5 + rng.uniform(-0.1, 0.1, sites.shape)) * a
    theta = math.radians(109.47)
    x = np.zeros((3 * nmol, 3))
    for w in range(nmol):
        e1 = _unit(rng.normal(size=3))
        e2 = _unit(np.cross(e1, _unit(rng.normal(size=3))))
        h1 = o[w] + 1.0 * e1
        h2 = o[w] + 1.0 * (math.cos(theta) * e1 + math.sin(theta) * e2)
        x[3 * w], x[3 * w + 1], x[3 * w + 2] = o[w], h1, h2
    n = 3 * nmol
    tidx = np.tile([0, 1, 1], nmol).astype(np.int32)
    q = np.tile([-0.8476, 0.4238, 0.4238], nmol)
    mass = np.tile([M_O, M_H, M_H], nmol)
    bonds = np.array([(3 * w, 3 * w + b) for w in range(nmol) for b in (1, 2)], np.uint32)
    ang = np.array([(3 * w + 1, 3 * w, 3 * w + 2) for w in range(nmol)], np.uint32)
    nb = _graph(n, bonds)
    off, lst, _ = exclusions(n, nb, depth=2)
    eps_o = 0.650 / 4.184
    pe = np.array([[eps_o, 0.0], [0.0, 0.0]])
    ps = np.array([[3.166, 1.0], [1.0, 1.0]])
    ff = ForceField(type_index=tidx, charge=q, mass=mass, pair_eps=pe, pair_sigma=ps, bond_ij=bonds,
                    bond_k_r0=np.tile([450.0, 1.0], (len(bonds), 1)), angle_ijk=ang,
                    angle_kt_theta0=np.tile([55.0, theta], (len(ang), 1)), excl_offset=off, excl_list=lst,
                    element=np.tile([8, 1, 1], nmol).astype(np.int32))
    cell = np.array([0, 0, 0, L, 0, 0, 0, L, 0, 0, 0, L], float)
    return ff, x, cell


def tile(ff: ForceField, x, cell, reps=(2, 2, 2)):
    """A periodic system repeated reps[0] x reps[1] x reps[2] times: the same periodic structure at a larger period
    (every copy keeps its molecules' unwrapped coordinates). Returns (force field, positions, cell)."""
    x = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    c = np.asarray(cell, dtype=np.float64).reshape(12)
    n = ff.natoms
    edges = c[3:].reshape(3, 3)
    shifts = [i * edges[0] + j * edges[1] + k * edges[2] for i in range(reps[0]) for j in range(reps[1]) for k in range(reps[2])]
    m = len(shifts)

    def idx(a):
        a = np.asarray(a, dtype=np.int64)
        return np.concatenate([a + q * n for q in range(m)]).astype(np.uint32) if len(a) else a.astype(np.uint32)

    def rep(a):
        return None if a is None else np.concatenate([np.asarray(a)] * m)

    off = np.asarray(ff.excl_offset, dtype=np.int64)
    lst = np.asarray(ff.excl_list, dtype=np.int64)
    excl_off = np.concatenate([off[:-1] + q * len(lst) for q in range(m)] + [[m * len(lst)]]).astype(np.uint32)
    excl_list = np.concatenate([lst + q * n for q in range(m)]).astype(np.uint32) if len(lst) else lst.astype(np.uint32)
    big = ForceField(type_index=rep(ff.type_index), charge=rep(ff.charge), mass=rep(ff.mass), pair_eps=ff.pair_eps, pair_sigma=ff.pair_sigma,
                     bond_ij=idx(ff.bond_ij), bond_k_r0=rep(ff.bond_k_r0), angle_ijk=idx(ff.angle_ijk), angle_kt_theta0=rep(ff.angle_kt_theta0),
                     dihedral_ijkl=idx(ff.dihedral_ijkl), dihedral_v_delta=rep(ff.dihedral_v_delta), dihedral_n=rep(ff.dihedral_n),
                     improper_ijkl=idx(ff.improper_ijkl), improper_v_delta=rep(ff.improper_v_delta), improper_n=rep(ff.improper_n),
                     pair14_ij=idx(ff.pair14_ij), pair14_lj=rep(ff.pair14_lj), pair14_coul=rep(ff.pair14_coul), lj14=ff.lj14, coul14=ff.coul14,
                     excl_offset=excl_off, excl_list=excl_list, fene_ij=idx(ff.fene_ij), fene_k_r0_eps_sigma=rep(ff.fene_k_r0_eps_sigma),
                     lj_shift=ff.lj_shift, model_cutoff=ff.model_cutoff, element=rep(ff.element))
    xb = np.concatenate([x + s_ for s_ in shifts])
    cb = c.copy()
    cb[3:6] *= reps[0]
    cb[6:9] *= reps[1]
    cb[9:12] *= reps[2]
    return big, xb, cb



# --- cis-1,4-polyisoprene and graphene (the rubber configurations) ---------------------------------------------------
# OPLS-AA-style classes: CT sp3 carbon, CM sp2 carbon, HC hydrogen on sp3 carbon, HM hydrogen on sp2 carbon, CG graphene
# carbon (neutral; eps 0.293 kJ/mol, sigma 3.55 Å).
_PI_LJ = {"CT": (0.066, 3.50), "CM": (0.076, 3.55), "HC": (0.030, 2.50), "HM": (0.030, 2.42), "CG": (0.293 / 4.184, 3.55)}
_PI_BOND = {("CT", "CT"): (268.0, 1.529), ("CT", "CM"): (317.0, 1.510), ("CM", "CM"): (549.0, 1.340), ("CT", "HC"): (340.0, 1.090),
            ("CM", "HM"): (340.0, 1.080), ("CG", "CG"): (469.0, 1.420)}
_PI_ANGLE = {("CT", "CT", "CM"): (63.0, 111.1), ("CT", "CT", "HC"): (37.5, 110.7), ("HC", "CT", "CM"): (35.0, 109.5),
             ("HC", "CT", "HC"): (33.0, 107.8), ("CT", "CM", "CM"): (70.0, 122.0), ("CT", "CM", "CT"): (70.0, 116.0),
             ("CM", "CM", "HM"): (35.0, 120.0), ("HM", "CM", "CT"): (35.0, 118.0), ("CG", "CG", "CG"): (63.0, 120.0)}
# Fourier V1, V2, V3 as in the polystyrene table; torsions not listed carry no term
_PI_TORS = {("CT", "CM", "CM", "CT"): (0.0, 14.0, 0.0), ("CT", "CM", "CM", "HM"): (0.0, 14.0, 0.0),
            ("CM", "CM", "CT", "CT"): (0.346, 0.405, -0.940), ("CM", "CM", "CT", "HC"): (0.0, 0.0, -0.372),
            ("CM", "CT", "CT", "CM"): (1.740, -0.157, 0.279), ("CM", "CT", "CT", "HC"): (0.0, 0.0, 0.300),
            ("HC", "CT", "CT", "HC"): (0.0, 0.0, 0.300), ("CT", "CM", "CT", "HC"): (0.0, 0.0, 0.300),
            ("HM", "CM", "CT", "HC"): (0.0, 0.0, 0.300), ("HM", "CM", "CT", "CT"): (0.0, 0.0, 0.300),
            ("CG", "CG", "CG", "CG"): (0.0, 7.250, 0.0)}
# charges per position in the unit: CH2 -0.12 / H +0.06, quaternary sp2 C 0, =CH- -0.115 / H +0.115, CH3 -0.18 / H +0.06
_PI_UNIT_Q = [-0.12, 0.0, -0.115, -0.12, -0.18, 0.06, 0.06, 0.115, 0.06, 0.06, 0.06, 0.06, 0.06]
_PI_CLASSES = ["CT", "CM", "HC", "HM", "CG"]
# one repeat unit -CH2-C(CH3)=CH-CH2-: C1 C2 C3 C4 C5(methyl) H1 H1 H3 H4 H4 H5 H5 H5
_PI_UNIT = ["CT", "CM", "CM", "CT", "CT", "HC", "HC", "HM", "HC", "HC", "HC", "HC", "HC"]
_PI_UNIT_BONDS = [(0, 1), (1, 2), (2, 3), (1, 4), (0, 5), (0, 6), (2, 7), (3, 8), (3, 9), (4, 10), (4, 11), (4, 12)]


def _topology_terms(cls: list[str], bonds: np.ndarray, bond_t: dict, angle_t: dict, tors_t: dict):
    """Bond, angle and torsion parameters for a molecule from per-atom classes (bonds given); torsions without an
    entry carry no term."""
    n = len(cls)
    nb = _graph(n, bonds)
    bk = np.array([_key_sym(bond_t, (cls[i], cls[j])) for i, j in bonds], float).reshape(-1, 2)
    ang = angles_from_bonds(nb)
    ak = np.array([(lambda p: (p[0], math.radians(p[1])))(_key_sym(angle_t, (cls[i], cls[j], cls[k]))) for i, j, k in ang],
                  float).reshape(-1, 2)
    d_ijkl, d_vd, d_n = [], [], []
    for i, j, k, l in dihedrals_from_bonds(nb, bonds):
        v = _key_sym(tors_t, (cls[i], cls[j], cls[k], cls[l]))
        if v is None:
            continue
        for nn, (vv, delta) in enumerate(((v[0] / 2, 0.0), (v[1] / 2, math.pi), (v[2] / 2, 0.0)), start=1):
            if vv != 0.0:
                d_ijkl.append((i, j, k, l))
                d_vd.append((vv, delta))
                d_n.append(nn)
    off, lst, p14 = exclusions(n, nb)
    return dict(bond_ij=bonds, bond_k_r0=bk, angle_ijk=ang, angle_kt_theta0=ak, dihedral_ijkl=np.array(d_ijkl, np.uint32).reshape(-1, 4),
                dihedral_v_delta=np.array(d_vd, float).reshape(-1, 2), dihedral_n=np.array(d_n, np.int32), pair14_ij=p14,
                excl_offset=off, excl_list=lst)


def _replicate(template: dict, natoms: int, copies: int) -> dict:
    """The terms of `copies` copies of a molecule of `natoms` atoms, each shifted by natoms in index."""
    out = {}
    for k in ("bond_ij", "angle_ijk", "dihedral_ijkl", "improper_ijkl", "pair14_ij"):
        a = np.asarray(template.get(k, np.zeros((0, 2), np.uint32)), dtype=np.int64)
        out[k] = (a[None] + natoms * np.arange(copies)[:, None, None]).reshape(-1, a.shape[1]).astype(np.uint32) if a.size else a.astype(np.uint32)
    for k in ("bond_k_r0", "angle_kt_theta0", "dihedral_v_delta", "dihedral_n", "improper_v_delta", "improper_n"):
        a = np.asarray(template.get(k, np.zeros((0,))))
        out[k] = np.concatenate([a] * copies) if a.size else a
    off = np.asarray(template["excl_offset"], dtype=np.int64)
    lst = np.asarray(template["excl_list"], dtype=np.int64)
    out["excl_offset"] = np.concatenate([off[:-1] + q * len(lst) for q in range(copies)] + [[copies * len(lst)]]).astype(np.uint32)
    out["excl_list"] = (lst[None] + natoms * np.arange(copies)[:, None]).reshape(-1).astype(np.uint32)
    return out


def _concat_terms(parts: list[tuple[dict, int]]) -> dict:
    """Joins the terms of molecules placed one after another (each with its atom count)."""
    out, base, ebase = {}, 0, 0
    keys_idx = ("bond_ij", "angle_ijk", "dihedral_ijkl", "improper_ijkl", "pair14_ij")
    keys_val = ("bond_k_r0", "angle_kt_theta0", "dihedral_v_delta", "dihedral_n", "improper_v_delta", "improper_n")
    acc = {k: [] for k in keys_idx + keys_val}
    offs, lsts = [], []
    for t, n in parts:
        for k in keys_idx:
            a = np.asarray(t.get(k, np.zeros((0, 2))), dtype=np.int64)
            if a.size:
                acc[k].append(a + base)
        for k in keys_val:
            a = np.asarray(t.get(k, np.zeros((0,))))
            if a.size:
                acc[k].append(a)
        off = np.asarray(t["excl_offset"], dtype=np.int64)
        offs.append(off[:-1] + ebase)
        lsts.append(np.asarray(t["excl_list"], dtype=np.int64) + base)
        ebase += int(off[-1])
        base += n
    for k in keys_idx:
        w = {"bond_ij": 2, "pair14_ij": 2, "angle_ijk": 3}.get(k, 4)
        out[k] = np.concatenate(acc[k]).astype(np.uint32) if acc[k] else np.zeros((0, w), np.uint32)
    for k in keys_val:
        out[k] = np.concatenate(acc[k]) if acc[k] else np.zeros((0,))
    out["excl_offset"] = np.concatenate(offs + [[ebase]]).astype(np.uint32)
    out["excl_list"] = np.concatenate(lsts).astype(np.uint32)
    return out


def _pi_chain_terms(units: int) -> tuple[list[str], dict]:
    """Classes and terms of one cis-1,4-polyisoprene chain of `units` repeat units (13 atoms each, chain ends open)."""
    cls = _PI_UNIT * units
    bonds = []
    for u in range(units):
        o = 13 * u
        bonds += [(o + a, o + b) for a, b in _PI_UNIT_BONDS]
        if u > 0:
            bonds.append((o - 13 + 3, o))   # C4 of the previous unit to C1
    terms = _topology_terms(cls, np.array(bonds, np.uint32), _PI_BOND, _PI_ANGLE, _PI_TORS)
    # impropers holding the sp2 carbons planar: C2 (C1, C3; C5) and C3 (C2, C4; H), v [1 + cos(2 phi - pi)], v = 7.5
    imp = []
    for u in range(units):
        o = 13 * u
        imp += [(o, o + 2, o + 1, o + 4), (o + 1, o + 3, o + 2, o + 7)]
    terms["improper_ijkl"] = np.array(imp, np.uint32)
    terms["improper_v_delta"] = np.tile([7.5, math.pi], (len(imp), 1))
    terms["improper_n"] = np.full(len(imp), 2, np.int32)
    return cls, terms


class _Occupancy:
    """Counts of placed heavy atoms on a periodic voxel grid, for steering chain growth away from occupied space."""

    def __init__(self, L: float, voxel: float = 2.2):
        self.n = max(4, int(L / voxel))
        self.h = L / self.n
        self.count = np.zeros((self.n,) * 3, np.int32)
        self.L = L

    def _idx(self, p):
        return (np.floor(np.mod(p, self.L) / self.h).astype(np.int64)) % self.n

    def add(self, p):
        i = self._idx(np.asarray(p).reshape(-1, 3))
        np.add.at(self.count, (i[:, 0], i[:, 1], i[:, 2]), 1)

    def crowding(self, p):
        """Occupied counts in the 3 x 3 x 3 voxels around each point of p (... x 3)."""
        shp = p.shape[:-1]
        i = self._idx(p.reshape(-1, 3))
        s = np.zeros(len(i), np.int64)
        for d in ((a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)):
            j = (i + np.array(d)) % self.n
            s += self.count[j[:, 0], j[:, 1], j[:, 2]]
        return s.reshape(shp)


def _nerf_v(a, b, c, bond, angle, torsion):
    """Vectorised _nerf: rows of a, b, c (m x 3); bond, angle, torsion scalars or (m,) arrays."""
    bc = c - b
    bc /= np.linalg.norm(bc, axis=-1, keepdims=True)
    nrm = np.cross(b - a, bc)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    m2 = np.cross(nrm, bc)
    d0 = -bond * np.cos(angle)
    d1 = bond * np.sin(angle) * np.cos(torsion)
    d2 = bond * np.sin(angle) * np.sin(torsion)
    return c + bc * np.asarray(d0)[..., None] + m2 * np.asarray(d1)[..., None] + nrm * np.asarray(d2)[..., None]


def _grow_pi_chains(chains: int, units: int, L: float, rng, occ: _Occupancy, tries: int = 8) -> np.ndarray:
    """Positions (chains, 13 units, 3) of cis-1,4-polyisoprene chains grown together in a periodic cube: every backbone
    step takes, of `tries` torsions drawn from the allowed states (cis about the double bond), the least crowded."""
    nb = 4 * units
    bb = np.zeros((chains, nb, 3))
    blen = {0: 1.529, 1: 1.510, 2: 1.340, 3: 1.510}                 # bond into backbone atom k, by k % 4
    bang = {0: 111.1, 1: 111.1, 2: 122.0, 3: 122.0}                 # angle at atom k - 1, by k % 4
    # seeds: a random point and a random zig-zag of three atoms
    p0 = rng.uniform(0, L, (chains, 3))
    d1 = rng.normal(size=(chains, 3))
    d1 /= np.linalg.norm(d1, axis=1, keepdims=True)
    perp = np.cross(d1, rng.normal(size=(chains, 3)))
    perp /= np.linalg.norm(perp, axis=1, keepdims=True)
    bb[:, 0] = p0
    bb[:, 1] = p0 + 1.510 * d1
    t = math.radians(122.0)
    bb[:, 2] = bb[:, 1] + 1.340 * (-math.cos(t) * d1 + math.sin(t) * perp)
    prev = bb[:, 0] - 1.529 * (math.cos(math.pi - math.radians(111.1)) * d1 + math.sin(math.pi - math.radians(111.1)) * perp)
    occ.add(bb[:, :3])
    for k in range(3, nb):
        a = bb[:, k - 3] if k >= 3 else prev
        centre = (k - 2) % 4                                         # the bond (k-2, k-1) the torsion turns about
        if centre == 1:
            choices = np.zeros((chains, tries))                      # cis about C2=C3
        elif centre == 3:
            choices = rng.choice([math.pi, math.pi / 3, -math.pi / 3], size=(chains, tries), p=[0.6, 0.2, 0.2])
        else:
            choices = rng.choice([math.pi, 2 * math.pi / 3, -2 * math.pi / 3], size=(chains, tries))
        choices = choices + rng.normal(0, math.radians(12), size=(chains, tries)) * (centre != 1)
        A = np.repeat(a[:, None], tries, 1).reshape(-1, 3)
        B = np.repeat(bb[:, k - 2, None], tries, 1).reshape(-1, 3)
        Cc = np.repeat(bb[:, k - 1, None], tries, 1).reshape(-1, 3)
        cand = _nerf_v(A, B, Cc, blen[k % 4], math.radians(bang[k % 4]), choices.reshape(-1)).reshape(chains, tries, 3)
        crowd = occ.crowding(cand) + rng.uniform(0, 0.5, (chains, tries))
        pick = np.argmin(crowd, axis=1)
        bb[:, k] = cand[np.arange(chains), pick]
        occ.add(bb[:, k])
    # side atoms per unit: methyl C5 and the hydrogens, from the local backbone geometry
    X = np.zeros((chains, units, 13, 3))
    X[:, :, 0:4] = bb.reshape(chains, units, 4, 3)
    c1, c2, c3, c4 = (X[:, :, q] for q in range(4))
    # the neighbours across the unit boundaries; at the chain ends, stand-ins where the chain would continue
    end = _nerf_v(bb[:, -3], bb[:, -2], bb[:, -1], 1.529, math.radians(111.1), math.pi)
    prev_c4 = np.concatenate([prev[:, None], c4[:, :-1]], axis=1)
    next_c1 = np.concatenate([c1[:, 1:], end[:, None]], axis=1)

    def unit(v):
        return v / np.linalg.norm(v, axis=-1, keepdims=True)

    def planar(centre, n1, n2, length):
        return centre + length * unit(-(unit(n1 - centre) + unit(n2 - centre)))

    def tetra2(centre, n1, n2, length):
        u1, u2 = unit(n1 - centre), unit(n2 - centre)
        bis, nrm = unit(-(u1 + u2)), unit(np.cross(u1, u2))
        ang = math.radians(54.75)
        return (centre + length * unit(bis * math.cos(ang) + nrm * math.sin(ang)), centre + length * unit(bis * math.cos(ang) - nrm * math.sin(ang)))

    X[:, :, 4] = planar(c2, c1, c3, 1.510)                         # methyl carbon in the double bond's plane
    X[:, :, 5], X[:, :, 6] = tetra2(c1, prev_c4, c2, 1.090)
    X[:, :, 7] = planar(c3, c2, c4, 1.080)
    X[:, :, 8], X[:, :, 9] = tetra2(c4, c3, next_c1, 1.090)
    c5 = X[:, :, 4]
    ax = unit(c5 - c2)
    ref = unit(np.cross(ax, c1 - c2))
    ref2 = np.cross(ax, ref)
    for q, phi in enumerate((0.0, 2 * math.pi / 3, 4 * math.pi / 3)):
        d = ax * math.cos(math.radians(180 - 109.5)) + math.sin(math.radians(180 - 109.5)) * (ref * math.cos(phi) + ref2 * math.sin(phi))
        X[:, :, 10 + q] = c5 + 1.090 * unit(d)
    occ.add(X[:, :, 4])
    return X


def _pair_tables(classes: list[str]):
    eps = np.array([_PI_LJ[c][0] for c in classes])
    sig = np.array([_PI_LJ[c][1] for c in classes])
    return np.sqrt(np.outer(eps, eps)), np.sqrt(np.outer(sig, sig))


def _pi_forcefield(n_chain_atoms: list[int], units_per_chain: int, extra: list[tuple[list[str], dict, int]] | None = None) -> ForceField:
    """The force field of the given polyisoprene chains (one template repeated) followed by other molecules
    (classes, terms, atoms)."""
    cls1, t1 = _pi_chain_terms(units_per_chain)
    parts, cls = [], []
    nchains = len(n_chain_atoms)
    rep = _replicate(t1, len(cls1), nchains)
    parts.append((rep, len(cls1) * nchains))
    cls += cls1 * nchains
    for ecls, eterms, en in extra or []:
        parts.append((eterms, en))
        cls += ecls
    terms = _concat_terms(parts)
    tidx = np.array([_PI_CLASSES.index(c) for c in cls], np.int32)
    pe, ps = _pair_tables(_PI_CLASSES)
    q = np.concatenate([np.tile(_PI_UNIT_Q, units_per_chain * nchains), np.zeros(len(cls) - 13 * units_per_chain * nchains)])
    mass = np.array([M_C if c in ("CT", "CM", "CG") else M_H for c in cls])
    el = np.array([6 if c in ("CT", "CM", "CG") else 1 for c in cls], np.int32)
    return ForceField(type_index=tidx, charge=q, mass=mass, pair_eps=pe, pair_sigma=ps, lj14=0.5, coul14=0.5, element=el, **terms)


def polyisoprene_melt(chains: int, units: int = 100, density: float = 0.91, seed: int = 1) -> tuple[ForceField, np.ndarray, np.ndarray]:
    """cis-1,4-polyisoprene, `chains` x `units` repeat units of 13 atoms (-CH2-C(CH3)=CH-CH2-: 5 C + 8 H; chain ends
    open), OPLS-AA-style (geometric mixing, 1-4 at 0.5; CH2 -0.12 / H +0.06, =CH- -0.115 / +0.115 on its H, the
    quaternary sp2 C 0, CH3 -0.18 / H +0.06: every unit neutral), grown at `density` g/cm^3 in a cubic periodic box.
    Returns (force field, x [n, 3], cell[12]); the overlaps a dense growth leaves are pushed off on the device."""
    rng = np.random.default_rng(seed)
    mass_unit = 5 * M_C + 8 * M_H
    L = (chains * units * mass_unit / (density * NA) * 1e24) ** (1.0 / 3.0)
    occ = _Occupancy(L)
    X = _grow_pi_chains(chains, units, L, rng, occ)
    ff = _pi_forcefield([13 * units] * chains, units)
    cell = np.array([0, 0, 0, L, 0, 0, 0, L, 0, 0, 0, L], float)
    return ff, X.reshape(-1, 3), cell


def graphene_sheet(lx: float = 100.0, ly: float = 100.0, cc: float = 1.42) -> tuple[np.ndarray, np.ndarray]:
    """A flat honeycomb flake in the xy plane (rectangular cell sqrt(3) cc x 3 cc with four atoms, repeated to about
    lx x ly, edges left open), and its C-C bonds. Returns (positions [n, 3], bonds [m, 2])."""
    from scipy.spatial import cKDTree
    a, h = math.sqrt(3.0) * cc, 3.0 * cc
    nx, ny = max(3, int(round(lx / a))), max(2, int(round(ly / h)))
    basis = np.array([[0, 0], [a / 2, cc / 2], [a / 2, 1.5 * cc], [0, 2 * cc]])
    ij = np.array([(i, j) for i in range(nx) for j in range(ny)], float)
    xy = (ij[:, None, :] * np.array([a, h]) + basis[None]).reshape(-1, 2)
    x = np.concatenate([xy, np.zeros((len(xy), 1))], axis=1)
    pairs = np.array(sorted(cKDTree(x).query_pairs(1.15 * cc)), np.uint32).reshape(-1, 2)
    return x, pairs


def rubber_composite(natoms: int = 1_000_000, sheets: int = 4, units: int = 200, density: float = 0.91, seed: int = 1,
                     sheet_size: float = 100.0) -> tuple[ForceField, np.ndarray, np.ndarray]:
    """cis-1,4-polyisoprene chains of `units` repeat units packed around `sheets` neutral graphene flakes (about
    sheet_size x sheet_size Å, eps 0.293 kJ/mol, sigma 3.55 Å, bonded with angle and planarity terms) at `density`
    g/cm^3, about `natoms` atoms in all. The sheets lie flat at evenly spaced heights, alternately centred on two
    diagonal points of the cell; the chains grow around them. Returns (force field, x, cell)."""
    rng = np.random.default_rng(seed)
    gx, gb = graphene_sheet(sheet_size, sheet_size)
    ng = len(gx)
    chains = max(1, int(round((natoms - sheets * ng) / (13 * units))))
    mass = chains * units * (5 * M_C + 8 * M_H) + sheets * ng * M_C
    L = (mass / (density * NA) * 1e24) ** (1.0 / 3.0)
    occ = _Occupancy(L)
    sheet_x = []
    centre = gx[:, :2].mean(0)
    for s in range(sheets):
        c2 = (np.array([0.25, 0.25]) if s % 2 == 0 else np.array([0.75, 0.75])) * L
        z = (s + 0.5) * L / sheets
        p = gx.copy()
        p[:, :2] += c2 - centre
        p[:, 2] = z
        sheet_x.append(p)
        occ.add(p)
        occ.add(p + np.array([0, 0, 1.7]))    # keep chains a van der Waals radius off the faces
        occ.add(p - np.array([0, 0, 1.7]))
    X = _grow_pi_chains(chains, units, L, rng, occ)
    # graphene terms: bonds, angles, ring torsions (planarity), no charges
    gcls = ["CG"] * ng
    gterms = _topology_terms(gcls, gb, _PI_BOND, _PI_ANGLE, _PI_TORS)
    gterms_all = _replicate(gterms, ng, sheets)
    ff = _pi_forcefield([13 * units] * chains, units, extra=[(gcls * sheets, gterms_all, ng * sheets)])
    x = np.concatenate([X.reshape(-1, 3)] + sheet_x)
    cell = np.array([0, 0, 0, L, 0, 0, 0, L, 0, 0, 0, L], float)
    return ff, x, cell


def push_off(ff: ForceField, x, cell, energy_kw: dict, temperature: float = 300.0, steps: int = 600,
             caps=(5.0, 20.0, 100.0, 500.0), log=None) -> np.ndarray:
    """Removes the overlaps a dense growth leaves: FP64 Langevin dynamics (dt 0.5 fs) under an LJ force cap raised stage
    by stage with Coulomb off, then one stage at the last cap with Coulomb on (the reference's relax push-off does the
    same with its force caps). energy_kw: the EnergyOptions fields of the run (cut-off, electrostatics ...). Returns x."""
    from .engine import DynamicsOptions, EnergyOptions, Evaluator
    stages = [(c, False) for c in caps] + [(caps[-1], True)]
    ev = None
    for k, (cap, coul) in enumerate(stages):
        eo = EnergyOptions(**{**energy_kw, "coulomb": coul and energy_kw.get("coulomb", True), "precision": "double", "force_cap": cap})
        o = DynamicsOptions(dt=0.5, steps=steps, temperature=temperature, thermostat="langevin", tau_t=20.0, thermo_every=steps,
                            seed=7 + k, energy=eo, new_velocities=True)
        if ev is None:
            ev = Evaluator(ff, eo)
        else:
            ev.set_options(eo)
        out = ev.run(x, cell, o)
        x = out["x"]
        if log:
            log(f"push-off cap {cap:6.0f} coulomb {coul}: T {out['thermo'][-1]['temperature']:.0f} K, E {out['thermo'][-1]['potential']:.0f} kcal/mol")
    ev.close()
    return x


def push_off_batch(ffs: list, xs: list, cells: list, energy_kw: dict, temperature: float = 300.0, steps: int = 600,
                   caps=(5.0, 20.0, 100.0, 500.0), log=None) -> list:
    """push_off for independent systems at once: every stage one run_batch over all of them."""
    from .engine import DynamicsOptions, EnergyOptions, Evaluator, run_batch
    stages = [(c, False) for c in caps] + [(caps[-1], True)]
    evs = []
    xs = [np.asarray(x, dtype=np.float64).reshape(-1, 3) for x in xs]
    for k, (cap, coul) in enumerate(stages):
        eo = EnergyOptions(**{**energy_kw, "coulomb": coul and energy_kw.get("coulomb", True), "precision": "double", "force_cap": cap})
        opts = [DynamicsOptions(dt=0.5, steps=steps, temperature=temperature, thermostat="langevin", tau_t=20.0, thermo_every=steps,
                                seed=7 + k + 1000 * r, energy=eo, new_velocities=True) for r in range(len(ffs))]
        if not evs:
            evs = [Evaluator(ff, eo) for ff in ffs]
        else:
            for ev in evs:
                ev.set_options(eo)
        out = run_batch(evs, xs, cells, opts)
        xs = [o["x"] for o in out]
        if log:
            log(f"push-off cap {cap:6.0f} coulomb {coul}: {len(ffs)} systems, mean T "
                f"{np.mean([o['thermo'][-1]['temperature'] for o in out]):.0f} K")
    for ev in evs:
        ev.close()
    return xs
