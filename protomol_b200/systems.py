"""Seeded synthetic molecular systems for the nonbonded force path.

Every system the benchmarks and parity tests use is generated here from a
seed, so the CPU reference, the CPU restatement and the GPU kernels all see
bit-identical inputs.  The layout mirrors what ProtoMol's ``buildTopology``
produces (``frontend/buildTopology.cpp``):

* charges are stored pre-scaled by sqrt(332.0636) = 18.2226123264
  (``buildTopology.cpp:148``, ``base/pmconstants.cpp:72``);
* the Lennard-Jones table holds, per type pair, {A, B, A14, B14} with the
  CHARMM combination rule of ``buildTopology.cpp:646-664``:
  r_ij = Rmin/2_i + Rmin/2_j, e_ij = sqrt(eps_i eps_j),
  A = r_ij^12 e_ij, B = 2 r_ij^6 e_ij;
* exclusions are added bonds first, then angles (1-3), then dihedrals (1-4)
  exactly as ``buildExclusionTable`` (``buildTopology.cpp:963-1010``) does,
  with ``ExclusionTable::add`` semantics (``topology/ExclusionTable.cpp``):
  the table keeps the first class seen for a pair, the look-up keeps the last.

Geometry of TIP3P water: O-H 0.9572 A, H-O-H 104.52 deg.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field

import numpy as np

SQRT_COULOMB_CONSTANT = 18.2226123264

EXCLUSION_NONE = 0
EXCLUSION_MODIFIED = 1
EXCLUSION_FULL = 2

# TIP3P
_OH = 0.9572
_HOH = math.radians(104.52)
_Q_O, _Q_H = -0.834, 0.417
_EPS_O, _RMIN2_O = 0.1521, 1.7682
_EPS_H, _RMIN2_H = 0.0, 0.2245
_M_O, _M_H = 15.9994, 1.008
# seeded liquid-like disorder of the water oxygens (A, per component); the
# 216-water box keeps its exact 6x6x6 lattice
WATER_JITTER = 0.1


@dataclass
class System:
    """One periodic (or vacuum) system in ProtoMol's GenericTopology terms."""

    name: str
    positions: np.ndarray          # (N, 3) float64, Angstrom
    scaled_charge: np.ndarray      # (N,) float64, q * 18.2226123264
    atom_type: np.ndarray          # (N,) int32
    molecule: np.ndarray           # (N,) int32
    mass: np.ndarray               # (N,) float64
    type_params: np.ndarray        # (T, 4) float64: eps, Rmin/2, eps14, Rmin14/2
    lj_table: np.ndarray           # (T, T, 4) float64: A, B, A14, B14
    exclusions: np.ndarray         # (E, 3) int32: a1 < a2, table class
    exclusion_check: np.ndarray    # (E,) int32: class returned by check()
    box: np.ndarray                # (4, 3) float64: e1, e2, e3, origin
    csf: float = 1.0               # coulombScalingFactor
    cell_size: float = 5.0
    periodic: bool = True
    bonds: list = field(default_factory=list)
    angles: list = field(default_factory=list)
    dihedrals: list = field(default_factory=list)

    @property
    def n_atoms(self) -> int:
        return int(self.positions.shape[0])

    @property
    def n_types(self) -> int:
        return int(self.type_params.shape[0])

    @property
    def box_lengths(self) -> np.ndarray:
        return np.array([self.box[0, 0], self.box[1, 1], self.box[2, 2]])

    def copy(self) -> "System":
        import copy
        return copy.deepcopy(self)

    # ---- binary interchange with the C restatement and the reference driver
    MAGIC = b"PMSYS001"

    def to_bytes(self) -> bytes:
        """Little-endian blob read by ``oracle/pmsys.h`` (pmsys_read)."""
        n, t, e = self.n_atoms, self.n_types, int(self.exclusions.shape[0])
        head = self.MAGIC + struct.pack("<iiii", n, t, e, 1 if self.periodic else 0)
        head += struct.pack("<12d", *np.asarray(self.box, np.float64).ravel())
        head += struct.pack("<dd", float(self.csf), float(self.cell_size))
        parts = [
            head,
            np.ascontiguousarray(self.positions, "<f8").tobytes(),
            np.ascontiguousarray(self.scaled_charge, "<f8").tobytes(),
            np.ascontiguousarray(self.atom_type, "<i4").tobytes(),
            np.ascontiguousarray(self.molecule, "<i4").tobytes(),
            np.ascontiguousarray(self.lj_table, "<f8").tobytes(),
            np.ascontiguousarray(self.exclusions, "<i4").tobytes(),
            np.ascontiguousarray(self.exclusion_check, "<i4").tobytes(),
        ]
        return b"".join(parts)

    def save(self, path: str) -> None:
        with open(path, "wb") as fh:
            fh.write(self.to_bytes())


# --------------------------------------------------------------------------
# topology helpers
# --------------------------------------------------------------------------

def lj_table_from_types(type_params: np.ndarray) -> np.ndarray:
    """CHARMM combination rule (``frontend/buildTopology.cpp:646-664``)."""
    eps, rmin, eps14, rmin14 = (type_params[:, k] for k in range(4))
    r = rmin[:, None] + rmin[None, :]
    e = np.sqrt(eps[:, None] * eps[None, :])
    r14 = rmin14[:, None] + rmin14[None, :]
    e14 = np.sqrt(eps14[:, None] * eps14[None, :])
    out = np.empty(r.shape + (4,), np.float64)
    out[..., 0] = r ** 12 * e
    out[..., 1] = 2.0 * r ** 6 * e
    out[..., 2] = r14 ** 12 * e14
    out[..., 3] = 2.0 * r14 ** 6 * e14
    return out


def build_exclusions(bonds, angles, dihedrals, scheme: str = "scaled1-4"):
    """Replays ``buildExclusionTable`` + ``ExclusionTable::add``.

    Returns (table (E,3) int32, check_class (E,) int32).
    """
    table = []
    index = {}
    last = {}

    def add(a, b, cls):
        if a > b:
            a, b = b, a
        if cls != EXCLUSION_NONE and a != b and (a, b) not in index:
            index[(a, b)] = len(table)
            table.append((a, b, cls))
        last[(a, b)] = cls

    if scheme == "none":
        return np.zeros((0, 3), np.int32), np.zeros((0,), np.int32)
    for a, b in bonds:
        add(a, b, EXCLUSION_FULL)
    if scheme != "1-2":
        for a, _, c in angles:
            add(a, c, EXCLUSION_FULL)
        if scheme != "1-3":
            for a, _, _, d in dihedrals:
                add(a, d, EXCLUSION_FULL if scheme == "1-4" else EXCLUSION_MODIFIED)
    tab = np.array(table, np.int32).reshape(-1, 3)
    chk = np.array([last[(a, b)] for a, b, _ in table], np.int32)
    return tab, chk


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotation matrices (Shoemake's quaternion method)."""
    u1, u2, u3 = rng.random((3, n))
    q = np.stack([
        np.sqrt(1 - u1) * np.sin(2 * np.pi * u2),
        np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
        np.sqrt(u1) * np.sin(2 * np.pi * u3),
        np.sqrt(u1) * np.cos(2 * np.pi * u3),
    ], axis=1)
    x, y, z, w = q.T
    r = np.empty((n, 3, 3))
    r[:, 0, 0] = 1 - 2 * (y * y + z * z)
    r[:, 0, 1] = 2 * (x * y - z * w)
    r[:, 0, 2] = 2 * (x * z + y * w)
    r[:, 1, 0] = 2 * (x * y + z * w)
    r[:, 1, 1] = 1 - 2 * (x * x + z * z)
    r[:, 1, 2] = 2 * (y * z - x * w)
    r[:, 2, 0] = 2 * (x * z - y * w)
    r[:, 2, 1] = 2 * (y * z + x * w)
    r[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return r


def _water_atoms(rng, oxygens: np.ndarray, jitter: float = 0.0) -> np.ndarray:
    """Rigid TIP3P waters with uniform random orientation; returns (3n, 3).

    ``jitter`` > 0 displaces each oxygen by N(0, jitter) per component
    (liquid-like disorder; on an exact lattice thousands of O-O pairs share
    bit-identical distances, which no liquid configuration has)."""
    n = oxygens.shape[0]
    if jitter > 0.0:
        oxygens = oxygens + rng.normal(0.0, jitter, oxygens.shape)
    half = 0.5 * _HOH
    local = np.array([
        [0.0, 0.0, 0.0],
        [_OH * math.sin(half), 0.0, _OH * math.cos(half)],
        [-_OH * math.sin(half), 0.0, _OH * math.cos(half)],
    ])
    rot = _random_rotations(rng, n)
    pos = oxygens[:, None, :] + np.einsum("nij,aj->nai", rot, local)
    return pos.reshape(-1, 3)


def _min_image(d: np.ndarray, lengths: np.ndarray) -> np.ndarray:
    return d - lengths * np.rint(d / lengths)


def _random_walk_chain(rng, n, lengths, start, bond=1.53, angle_deg=111.0,
                       min_sep=2.6, tries=64):
    """Self-avoiding-ish random-walk chain built with NeRF placement.

    Bond 1.53 A, bond angle 111 deg, uniformly random dihedrals; a dihedral is
    redrawn (up to ``tries`` times) while the new atom comes closer than
    ``min_sep`` to any earlier non-1-2/1-3/1-4 atom (minimal image).
    """
    theta = math.radians(angle_deg)
    pos = np.zeros((n, 3))
    pos[0] = start
    if n > 1:
        v = rng.normal(size=3)
        pos[1] = pos[0] + bond * v / np.linalg.norm(v)
    if n > 2:
        a = pos[1] - pos[0]
        a /= np.linalg.norm(a)
        p = rng.normal(size=3)
        p -= a * (p @ a)
        p /= np.linalg.norm(p)
        pos[2] = pos[1] + bond * (-a * math.cos(theta) + p * math.sin(theta))
    for k in range(3, n):
        a, b, c = pos[k - 3], pos[k - 2], pos[k - 1]
        bc = c - b
        bc /= np.linalg.norm(bc)
        nrm = np.cross(b - a, bc)
        nrm /= np.linalg.norm(nrm)
        m = np.stack([bc, np.cross(nrm, bc), nrm], axis=1)
        best, best_d = None, -1.0
        for _ in range(tries):
            phi = rng.uniform(0.0, 2 * math.pi)
            d2 = np.array([-bond * math.cos(theta),
                           bond * math.sin(theta) * math.cos(phi),
                           bond * math.sin(theta) * math.sin(phi)])
            cand = c + m @ d2
            if k > 3:
                dd = _min_image(pos[: k - 3] - cand, lengths)
                dmin = float(np.sqrt((dd * dd).sum(1)).min())
            else:
                dmin = 1e9
            if dmin > best_d:
                best, best_d = cand, dmin
            if dmin >= min_sep:
                break
        pos[k] = best
    return pos


def _chain_topology(n, offset=0):
    bonds = [(offset + k, offset + k + 1) for k in range(n - 1)]
    angles = [(offset + k, offset + k + 1, offset + k + 2) for k in range(n - 2)]
    dihedrals = [(offset + k, offset + k + 1, offset + k + 2, offset + k + 3)
                 for k in range(n - 3)]
    return bonds, angles, dihedrals


def _water_topology(first_atom, n_water):
    bonds, angles = [], []
    for w in range(n_water):
        o = first_atom + 3 * w
        bonds += [(o, o + 1), (o, o + 2)]
        angles.append((o + 1, o, o + 2))
    return bonds, angles


def _cubic_box(length: float) -> np.ndarray:
    return np.array([[length, 0, 0], [0, length, 0], [0, 0, length], [0, 0, 0]], np.float64)


def _assemble(name, chain_pos, chain_q, chain_params, water_pos, extra=None, *,
              box_len, csf, cell_size, scheme, periodic=True):
    """Order: chain atoms, then waters (O,H,H), then extra single ions."""
    n_chain = 0 if chain_pos is None else chain_pos.shape[0]
    n_water = 0 if water_pos is None else water_pos.shape[0] // 3
    types = [[_EPS_O, _RMIN2_O, _EPS_O, _RMIN2_O], [_EPS_H, _RMIN2_H, _EPS_H, _RMIN2_H]]
    pos, q, ty, mol, mass = [], [], [], [], []
    bonds, angles, dihedrals = [], [], []
    next_mol = 0
    if n_chain:
        pos.append(chain_pos)
        q.append(chain_q)
        base = len(types)
        types += [list(p) for p in chain_params]
        ty.append(base + np.arange(n_chain))
        mol.append(np.full(n_chain, next_mol))
        mass.append(np.full(n_chain, 12.011))
        next_mol += 1
        b, a, d = _chain_topology(n_chain)
        bonds += b
        angles += a
        dihedrals += d
    if n_water:
        pos.append(water_pos)
        q.append(np.tile([_Q_O, _Q_H, _Q_H], n_water))
        ty.append(np.tile([0, 1, 1], n_water))
        mol.append(next_mol + np.repeat(np.arange(n_water), 3))
        mass.append(np.tile([_M_O, _M_H, _M_H], n_water))
        next_mol += n_water
        b, a = _water_topology(n_chain, n_water)
        bonds += b
        angles += a
    if extra:
        for (p, charge, eps, rmin2, m) in extra:
            pos.append(np.asarray(p, np.float64).reshape(1, 3))
            q.append(np.array([charge]))
            ty.append(np.array([len(types)]))
            types.append([eps, rmin2, eps, rmin2])
            mol.append(np.array([next_mol]))
            mass.append(np.array([m]))
            next_mol += 1
    tp = np.array(types, np.float64)
    # bonds listed chain first, then waters, matching a PSF in atom order
    excl, chk = build_exclusions(bonds, angles, dihedrals, scheme)
    return System(
        name=name,
        positions=np.concatenate(pos).astype(np.float64),
        scaled_charge=np.concatenate(q).astype(np.float64) * SQRT_COULOMB_CONSTANT,
        atom_type=np.concatenate(ty).astype(np.int32),
        molecule=np.concatenate(mol).astype(np.int32),
        mass=np.concatenate(mass).astype(np.float64),
        type_params=tp,
        lj_table=lj_table_from_types(tp),
        exclusions=excl,
        exclusion_check=chk,
        box=_cubic_box(box_len),
        csf=csf,
        cell_size=cell_size,
        periodic=periodic,
        bonds=bonds, angles=angles, dihedrals=dihedrals,
    )


def _lattice(n_side: int, length: float) -> np.ndarray:
    a = length / n_side
    g = (np.arange(n_side) + 0.5) * a - 0.5 * length
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)


# --------------------------------------------------------------------------
# the workloads
# --------------------------------------------------------------------------

def water_box_216(seed: int = 1) -> System:
    """216 TIP3P waters on a 6x6x6 lattice (3.1 A) in an 18.6 A cube.

    Cutoff 9 A, C2 switching 8->9 A, cell size 4.5 A; all intra-water pairs
    excluded (bonds + the H-H angle pair).
    """
    rng = np.random.default_rng(seed)
    oxy = _lattice(6, 18.6)
    water = _water_atoms(rng, oxy)
    return _assemble("water216", None, None, None, water, box_len=18.6, csf=1.0,
                     cell_size=4.5, scheme="1-3")


def oxygen_fluid_216(seed: int = 1) -> System:
    """The 216 oxygens of :func:`water_box_216` as a Lennard-Jones fluid (eps
    0.1521 kcal/mol, Rmin/2 1.7682 A, no charges, no molecules): dynamics
    without the SHAKE/RATTLE constraints that keep rigid waters together."""
    import dataclasses
    s = water_box_216(seed)
    o = np.flatnonzero(s.atom_type == 0)
    tp = s.type_params[:1].copy()
    return dataclasses.replace(
        s, name="oxygen216", positions=s.positions[o].copy(), scaled_charge=np.zeros(len(o)),
        atom_type=np.zeros(len(o), np.int32), molecule=np.arange(len(o), dtype=np.int32), mass=s.mass[o].copy(),
        type_params=tp, lj_table=lj_table_from_types(tp), exclusions=np.zeros((0, 3), np.int32),
        exclusion_check=np.zeros(0, np.int32), bonds=[], angles=[], dihedrals=[])


def ionic_fluid_216(seed: int = 1, charge: float = 0.4) -> System:
    """:func:`oxygen_fluid_216` with charges +-``charge`` e alternating
    (neutral): a fluid with electrostatics and no molecules."""
    import dataclasses
    s = oxygen_fluid_216(seed)
    q = np.where(np.arange(s.n_atoms) % 2 == 0, charge, -charge) * 18.2226123264
    return dataclasses.replace(s, name="ionic216", scaled_charge=q)


def chain_in_water_14281(seed: int = 2) -> System:
    """4,463 TIP3P waters + an 892-atom random-walk chain in a 52.3 A cube.

    Chain charges ~ N(0, 0.3 e) shifted to neutral, eps ~ U[0.05, 0.2],
    Rmin/2 ~ U[1.2, 2.1] (one type per chain atom, eps14 = eps/2),
    ``exclude scaled1-4`` with coulombScalingFactor 0.5, cell size 6 A.
    """
    return chain_in_water(892, 4463, 52.3, seed, lattice=18, name="chain14281")


def chain_in_water(n_chain: int, n_water: int, length: float, seed: int, lattice: int = 0,
                   name: str = "") -> System:
    """``n_chain``-atom random-walk chain in ``n_water`` TIP3P waters, cubic
    box ``length``; waters on a lattice of ``lattice``^3 sites (default: the
    smallest cube with room for the waters after the chain's neighbourhood
    is cleared)."""
    rng = np.random.default_rng(seed)
    lengths = np.full(3, length)
    if lattice <= 0:
        lattice = int(math.ceil((1.35 * n_water) ** (1.0 / 3.0)))
    chain = _random_walk_chain(rng, n_chain, lengths, start=rng.uniform(-5, 5, 3))
    q = rng.normal(0.0, 0.3, n_chain)
    q -= q.mean()
    eps = rng.uniform(0.05, 0.2, n_chain)
    rmin = rng.uniform(1.2, 2.1, n_chain)
    params = np.stack([eps, rmin, 0.5 * eps, rmin], axis=1)
    sites = _lattice(lattice, length)
    radius = 2.6
    while True:
        keep = np.ones(len(sites), bool)
        for k in range(0, n_chain, 64):
            d = _min_image(sites[:, None, :] - chain[None, k:k + 64, :], lengths)
            keep &= ((d * d).sum(-1) >= radius * radius).all(1)
        if keep.sum() >= n_water:
            break
        radius -= 0.1
    idx = np.sort(rng.choice(np.flatnonzero(keep), n_water, replace=False))
    water = _water_atoms(rng, sites[idx], jitter=WATER_JITTER)
    return _assemble(name or f"chain{n_chain + 3 * n_water}", chain, q, params, water, box_len=length,
                     csf=0.5, cell_size=6.0, scheme="scaled1-4")


def vacuum_chain_104(seed: int = 3) -> System:
    """104-atom vacuum random-walk chain, charges ~ N(0, 0.4 e),
    1-2/1-3 excluded, 1-4 scaled by 0.5 (csf 0.5, eps14 = eps/2)."""
    rng = np.random.default_rng(seed)
    n = 104
    chain = _random_walk_chain(rng, n, np.full(3, 1e6), start=np.zeros(3))
    q = rng.normal(0.0, 0.4, n)
    eps = rng.uniform(0.05, 0.2, n)
    rmin = rng.uniform(1.2, 2.1, n)
    params = np.stack([eps, rmin, 0.5 * eps, rmin], axis=1)
    sys_ = _assemble("vacuum104", chain, q, params, None, box_len=1e3, csf=0.5,
                     cell_size=6.0, scheme="scaled1-4", periodic=False)
    return sys_


def water_box(n_water: int, seed: int, density: float = 0.0334,
              cell_size: float = 4.5) -> System:
    """n_water TIP3P waters at ``density`` molecules/A^3 on a randomly thinned
    cubic lattice, random orientations (the batched-box workload)."""
    rng = np.random.default_rng(seed)
    length = (n_water / density) ** (1.0 / 3.0)
    n_side = int(math.ceil(n_water ** (1.0 / 3.0)))
    sites = _lattice(n_side, length)
    idx = np.sort(rng.choice(len(sites), n_water, replace=False))
    water = _water_atoms(rng, sites[idx], jitter=WATER_JITTER)
    return _assemble(f"water{n_water}", None, None, None, water, box_len=length,
                     csf=1.0, cell_size=cell_size, scheme="1-3")


def batched_water_boxes(count: int = 96, seed: int = 4, lo: int = 100, hi: int = 3000):
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, count)
    return [water_box(int(n), seed=1000 + k) for k, n in enumerate(sizes)]


def water_box_1m(seed: int = 5) -> System:
    """333,333 TIP3P waters + 1 Na+ (q +1, eps 0.0469, Rmin/2 1.3638) in a
    215.4 A cube (1,000,000 atoms), cell size 6 A."""
    rng = np.random.default_rng(seed)
    length = 215.4
    sites = _lattice(70, length)
    pick = rng.choice(len(sites), 333_334, replace=False)
    ion_site = sites[pick[0]]
    idx = np.sort(pick[1:])
    water = _water_atoms(rng, sites[idx], jitter=WATER_JITTER)
    return _assemble("water1M", None, None, None, water,
                     extra=[(ion_site, 1.0, 0.0469, 1.3638, 22.98977)],
                     box_len=length, csf=1.0, cell_size=6.0, scheme="1-3")


CHAIN_BOND = 1.53             # the random-walk chains' bond length (A)


def rattle_shake_constraints(system: System):
    """The bond constraints of SHAKE / RATTLE as
    buildRattleShakeBondConstraintList (topology/topologyutilities.cpp:
    782-860) builds them: every bond with its rest length (TIP3P O-H 0.9572 A,
    chain bonds 1.53 A), then for every angle whose two end atoms are light
    (mass < 5) the end-to-end distance sqrt(b^2 + c^2 - 2 b c cos(theta0))
    of its two bonds (the water's H-H).  Returns (atoms (K, 2) int32,
    rest lengths (K,) float64)."""
    m = np.asarray(system.mass)
    light = lambda a: m[a] < 5.0
    rest = {}
    atoms, lengths = [], []
    for a, b in system.bonds:
        r = _OH if (light(a) or light(b)) else CHAIN_BOND
        rest[(min(a, b), max(a, b))] = r
        atoms.append((a, b))
        lengths.append(r)
    for a1, a2, a3 in system.angles:
        if not (light(a1) and light(a3)):
            continue
        b = rest.get((min(a1, a2), max(a1, a2)))
        c = rest.get((min(a2, a3), max(a2, a3)))
        if b is None or c is None:
            continue
        atoms.append((a1, a3))
        lengths.append(math.sqrt(b * b + c * c - 2 * b * c * math.cos(_HOH)))
    return np.asarray(atoms, np.int32).reshape(-1, 2), np.asarray(lengths, np.float64)


def smooth_grid_size(length: float, spacing: float = 1.0) -> int:
    """Smallest 2^a 3^b 5^c >= ceil(length / spacing)."""
    n = max(4, int(math.ceil(length / spacing)))
    while True:
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1


def ewald_alpha(cutoff: float, accuracy: float = 1e-6) -> float:
    """The reference's default splitting parameter: bisection of
    erfc(alpha Rc)/Rc = accuracy (``NonbondedPMEwaldSystemForce.h:564-586``)."""
    alpha = 1.0
    while math.erfc(alpha * cutoff) / cutoff >= accuracy:
        alpha *= 2.0
    low, high = 0.0, alpha
    for _ in range(100):
        alpha = 0.5 * (low + high)
        if math.erfc(alpha * cutoff) / cutoff >= accuracy:
            low = alpha
        else:
            high = alpha
    return alpha


def perturbed(system: System, sigma: float, seed: int) -> System:
    """Copy with positions displaced by N(0, sigma) (fresh cell assignment)."""
    out = system.copy()
    rng = np.random.default_rng(seed)
    out.positions = out.positions + rng.normal(0.0, sigma, out.positions.shape)
    return out
