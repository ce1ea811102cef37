"""ProtoMol's input files for the nonbonded path: PSF (atoms, bonds, angles,
dihedrals, impropers), CHARMM parameter files (the NONBONDED section) and XYZ
positions, and the System the nonbonded forces read, built as
frontend/buildTopology.cpp builds a Topology from them:

* atom types by PSF type name, numbered in order of first appearance
  (buildTopology.cpp:124-128);
* scaled charges q * sqrt(332.0636) and masses (:132-133);
* the Lennard-Jones table by the CHARMM combination rule from the PAR
  nonbonded entries (:646-664; ``systems.lj_table_from_types``);
* molecules: the connected components of the bond / angle / dihedral /
  improper graph, numbered by their lowest atom (buildMoleculeTable,
  :733-905);
* the exclusion table of the ``exclude`` scheme (buildExclusionTable,
  :963-1010; ``systems.build_exclusions``).

The C++ adapter uses ProtoMol's own readers; this module serves Python users
of the library and writes the synthetic systems out for the reference.
"""
from __future__ import annotations

import re
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import systems
from .systems import SQRT_COULOMB_CONSTANT, System

# ------------------------------------------------------------------ readers


def _section_count(line: str) -> int:
    return int(line.split()[0])


def read_psf(path: str) -> dict:
    """X-PLOR / CHARMM PSF: the !NATOM records (number, segment, residue
    number, residue name, atom name, atom type, charge, mass) and the
    !NBOND / !NTHETA / !NPHI / !NIMPHI index lists (1-based in the file,
    0-based here)."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    out = {"atoms": [], "bonds": [], "angles": [], "dihedrals": [], "impropers": []}
    groups = {"!NBOND": ("bonds", 2), "!NTHETA": ("angles", 3), "!NPHI": ("dihedrals", 4),
              "!NIMPHI": ("impropers", 4)}
    k = 0
    while k < len(lines):
        line = lines[k]
        if "!NATOM" in line:
            n = _section_count(line)
            for rec in lines[k + 1:k + 1 + n]:
                f = rec.split()
                out["atoms"].append({"number": int(f[0]), "segment": f[1], "residue": int(f[2]),
                                     "residue_name": f[3], "name": f[4], "type": f[5],
                                     "charge": float(f[6]), "mass": float(f[7])})
            k += 1 + n
            continue
        key = next((g for g in groups if g in line), None)
        if key is not None:
            name, width = groups[key]
            n = _section_count(line)
            values: List[int] = []
            k += 1
            while len(values) < n * width and k < len(lines):
                values += [int(v) for v in lines[k].split()]
                k += 1
            out[name] = [tuple(v - 1 for v in values[i:i + width]) for i in range(0, n * width, width)]
            continue
        k += 1
    return out


# sigma -> Rmin/2 of the X-PLOR dialect (base/PAR.cpp:10)
SIGMA_XPLOR_TO_RMIN_HALF = 2.0 ** (-5.0 / 6.0)


def _is_real(tok: str) -> bool:
    try:
        float(tok)
        return True
    except ValueError:
        return False


def _par_records(path: str) -> List[List[str]]:
    """The PAR file as token lists: ``{...}`` comments (across lines), ``!``
    comments, ``*`` title lines and REMARK / SET lines removed
    (io/PARReader.cpp:120-190)."""
    records, depth = [], 0
    with open(path) as fh:
        for line in fh:
            kept = []
            for c in line:
                if c == "{":
                    depth += 1
                elif c == "}":
                    depth = max(depth - 1, 0)
                    kept.append(" ")
                elif depth == 0:
                    kept.append(c)
            text = "".join(kept).split("!")[0]
            toks = []
            for tok in text.split():
                if tok.startswith("*"):
                    break
                toks.append(tok)
            if toks and not toks[0].upper().startswith(("REMARK", "SET")):
                records.append(toks)
    return records


def read_par(path: str) -> dict:
    """The nonbonded part of a parameter file (io/PARReader.cpp:447-480), in
    file order:

    * NONBONDED records, either CHARMM28 (a NONBONDED section of
      ``type ignored epsilon Rmin/2 [ignored epsilon14 Rmin14/2]``) or X-PLOR
      (``NONBONDED type epsilon sigma epsilon14 sigma14`` per line, sigma
      converted to Rmin/2); the 1-4 values default to the normal ones;
    * NBFIX records ``type1 type2 A B [A14 B14]``.

    Epsilons are kept as magnitudes: CHARMM28 writes negative well depths and
    the combination rule takes sqrt(eps_i eps_j)."""
    nonbonded: List[Tuple[str, float, float, float, float]] = []
    nbfix: List[Tuple[str, str, float, float, float, float]] = []
    section = None
    for toks in _par_records(path):
        head = toks[0].upper()
        rest = toks[1:]
        sig = "".join("d" if _is_real(t) else "w" for t in rest)
        if head.startswith(("NONB", "NBON")) and sig == "wdddd":           # X-PLOR record
            e, s, e14, s14 = (float(t) for t in rest[1:])
            nonbonded.append((rest[0], abs(e), s * SIGMA_XPLOR_TO_RMIN_HALF, abs(e14), s14 * SIGMA_XPLOR_TO_RMIN_HALF))
            continue
        if head.startswith("NBFI") and sig in ("wwdd", "wwdddd"):
            v = [float(t) for t in rest[2:]]
            nbfix.append((rest[0], rest[1], v[0], v[1], v[-2], v[-1]))
            continue
        if head.startswith(("BOND", "ANGL", "THET", "DIHE", "PHI", "IMPR", "IMPH", "HBON", "END", "CMAP")):
            section = None
            continue
        if head.startswith(("NONB", "NBON")):
            section = "NONBONDED"
            continue
        if head.startswith("NBFI"):
            section = "NBFIX"
            continue
        sig = "".join("d" if _is_real(t) else "w" for t in toks)
        if section == "NONBONDED" and sig in ("wddd", "wdddddd"):
            v = [float(t) for t in toks[1:]]
            e14, r14 = (v[4], v[5]) if len(v) == 6 else (v[1], v[2])
            nonbonded.append((toks[0], abs(v[1]), v[2], abs(e14), r14))
        elif section == "NBFIX" and sig in ("wwdd", "wwdddd"):
            v = [float(t) for t in toks[2:]]
            nbfix.append((toks[0], toks[1], v[0], v[1], v[-2], v[-1]))
    return {"nonbonded": nonbonded, "nbfix": nbfix}


def _wildcard_regex(pattern: str) -> "re.Pattern":
    """The wildcards of equalWildcard (base/stringutilities.cpp:469): ``*``
    any characters, ``%`` one character, ``#`` digits, ``+`` one digit."""
    out = []
    for c in pattern:
        out.append({"*": ".*", "%": ".", "#": "[0-9]*", "+": "[0-9]"}.get(c, re.escape(c)))
    return re.compile("".join(out) + r"\Z")


def match_type(patterns: Sequence[str], name: str) -> int:
    """buildTopology's parameter look-up (buildTopology.cpp:608-618): the
    first exact match, else the first wildcard match, else -1."""
    best = -1
    for k, pat in enumerate(patterns):
        if pat == name:
            return k
        if best < 0 and any(c in pat for c in "*%#+") and _wildcard_regex(pat).match(name):
            best = k
    return best


def read_xyz(path: str) -> Tuple[List[str], np.ndarray]:
    """ProtoMol XYZ: the atom count, a comment line, then ``name x y z``."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    n = int(lines[0].split()[0])
    names, pos = [], np.zeros((n, 3))
    for i, rec in enumerate(lines[2:2 + n]):
        f = rec.split()
        names.append(f[0])
        pos[i] = [float(v) for v in f[1:4]]
    return names, pos


def read_pdb(path: str) -> Tuple[List[str], np.ndarray]:
    """Positions of the ATOM / HETATM records of a PDB file (atom name in
    columns 13-16, x y z in columns 31-54, as io/PDBReader.cpp reads them)."""
    names, pos = [], []
    with open(path) as fh:
        for line in fh:
            if line.startswith(("ATOM", "HETATM")):
                names.append(line[12:16].strip())
                pos.append((float(line[30:38]), float(line[38:46]), float(line[46:54])))
    return names, np.array(pos, np.float64).reshape(-1, 3)


def read_conf(path: str) -> dict:
    """The keywords of a ProtoMol configuration file that the nonbonded path
    reads (frontend/ProtoMolApp.cpp, frontend/inputValueDefinitions.h):
    posfile, psffile, parfile, exclude, boundaryConditions,
    cellBasisVector1..3, cellOrigin, cellsize; plus every ``force`` definition
    of the Integrator block as one string (continuation lines joined, ``#``
    comments removed, a leading ``time`` modifier dropped), level by level.
    Keys are lower-cased."""
    out: dict = {"forces": []}
    current = None
    with open(path) as fh:
        for raw in fh:
            line = raw.split("#")[0].strip()
            if not line:
                continue
            toks = line.replace("{", " { ").replace("}", " } ").split()
            head = toks[0].lower()
            if head == "force":
                body = toks[1:]
                if body and body[0].lower() == "time":
                    body = body[1:]
                current = " ".join(t for t in body if t not in "{}")
                out["forces"].append(current)
                continue
            if current is not None and toks[0].startswith("-"):
                current += " " + " ".join(t for t in toks if t not in "{}")
                out["forces"][-1] = current
                continue
            current = None
            if head in ("integrator", "level", "}", "{") or "{" in toks or "}" in toks:
                continue
            out[head] = toks[1:] if len(toks) > 2 else (toks[1] if len(toks) == 2 else "")
    return out


def load_conf(path: str) -> Tuple[System, List[str]]:
    """The System and the force definitions of a ProtoMol configuration file
    (paths in it relative to the file).  Positions come from posfile (XYZ or
    PDB); without cellBasisVectors the system is a vacuum one."""
    import os
    conf = read_conf(path)
    base = os.path.dirname(os.path.abspath(path))

    def file(key):
        if key not in conf:
            raise ValueError(f"{path}: no {key}")
        return os.path.join(base, conf[key])

    pos_file = file("posfile")
    names, pos = read_pdb(pos_file) if pos_file.lower().endswith(".pdb") else read_xyz(pos_file)
    psf = read_psf(file("psffile"))
    if len(names) != len(psf["atoms"]):
        raise ValueError(f"{pos_file} holds {len(names)} atoms, the PSF {len(psf['atoms'])}")
    periodic = str(conf.get("boundaryconditions", "vacuum")).lower() == "periodic"
    if all(f"cellbasisvector{k}" in conf for k in (1, 2, 3)):
        box = [[float(v) for v in conf[f"cellbasisvector{k}"]] for k in (1, 2, 3)]
        box.append([float(v) for v in conf.get("cellorigin", [0, 0, 0])])
    else:
        lo, hi = pos.min(0), pos.max(0)
        box = [[hi[0] - lo[0], 0, 0], [0, hi[1] - lo[1], 0], [0, 0, hi[2] - lo[2]], list(lo)]
    system = build_system(psf, read_par(file("parfile")), pos, box, float(conf.get("cellsize", 6.0)),
                          str(conf.get("exclude", "scaled1-4")), periodic=periodic,
                          name=os.path.basename(path))
    return system, conf["forces"]


# ------------------------------------------------------------------ topology


def molecules_of(n_atoms: int, *lists: Sequence[Tuple[int, ...]]) -> np.ndarray:
    """buildMoleculeTable: connected components of the graph whose edges join
    consecutive atoms of every bond, angle, dihedral and improper, numbered
    in the order of their lowest atom."""
    parent = list(range(n_atoms))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for lst in lists:
        for rec in lst:
            for a, b in zip(rec[:-1], rec[1:]):
                ra, rb = find(a), find(b)
                if ra != rb:
                    parent[max(ra, rb)] = min(ra, rb)
    mol = np.empty(n_atoms, np.int32)
    ids: Dict[int, int] = {}
    for i in range(n_atoms):
        r = find(i)
        if r not in ids:
            ids[r] = len(ids)
        mol[i] = ids[r]
    return mol


def build_system(psf: dict, par: dict, positions: np.ndarray, box, cell_size: float,
                 exclude: str = "scaled1-4", csf: float = 1.0, periodic: bool = True,
                 name: str = "psf") -> System:
    """The System of a PSF / PAR / positions triple, as buildTopology makes
    the GenericTopology (box: 4 x 3, the .conf's cellBasisVector1..3 and
    cellOrigin)."""
    atoms = psf["atoms"]
    n = len(atoms)
    type_index: Dict[str, int] = {}
    ty = np.empty(n, np.int32)
    for i, a in enumerate(atoms):
        ty[i] = type_index.setdefault(a["type"], len(type_index))
    type_list = sorted(type_index, key=type_index.get)
    patterns = [rec[0] for rec in par["nonbonded"]]
    rows = []
    for t in type_list:
        k = match_type(patterns, t)
        if k < 0:
            raise ValueError(f"no nonbonded parameters match atom type {t!r}")
        rows.append(par["nonbonded"][k][1:])
    tp = np.array(rows, np.float64).reshape(len(type_list), 4)
    table = systems.lj_table_from_types(tp)
    for t1, t2, a, b, a14, b14 in par.get("nbfix", []):          # buildTopology.cpp:671-719
        i, j = match_type(type_list, t1), match_type(type_list, t2)
        if i < 0:
            continue
        if j < 0:
            raise ValueError(f"no atom type matches the NBFIX pair {t1!r} - {t2!r}")
        table[i, j] = table[j, i] = (a, b, a14, b14)
    bonds, angles = list(psf["bonds"]), list(psf["angles"])
    dihedrals, impropers = list(psf["dihedrals"]), list(psf["impropers"])
    excl, chk = systems.build_exclusions(bonds, angles, dihedrals, exclude)
    return System(
        name=name,
        positions=np.ascontiguousarray(positions, np.float64),
        scaled_charge=np.array([a["charge"] for a in atoms], np.float64) * SQRT_COULOMB_CONSTANT,
        atom_type=ty,
        molecule=molecules_of(n, bonds, angles, dihedrals, impropers),
        mass=np.array([a["mass"] for a in atoms], np.float64),
        type_params=tp,
        lj_table=table,
        exclusions=excl,
        exclusion_check=chk,
        box=np.asarray(box, np.float64).reshape(4, 3),
        csf=csf,
        cell_size=cell_size,
        periodic=periodic,
        bonds=bonds, angles=angles, dihedrals=dihedrals,
    )


def load(psf_path: str, par_path: str, xyz_path: str, box, cell_size: float, exclude: str = "scaled1-4",
         csf: float = 1.0, periodic: bool = True) -> System:
    names, pos = read_xyz(xyz_path)
    psf = read_psf(psf_path)
    if len(names) != len(psf["atoms"]):
        raise ValueError(f"{xyz_path} holds {len(names)} atoms, {psf_path} {len(psf['atoms'])}")
    return build_system(psf, read_par(par_path), pos, box, cell_size, exclude, csf, periodic,
                        name=psf_path.rsplit("/", 1)[-1])


# ------------------------------------------------------------------ writers


def type_names(system: System) -> List[str]:
    return [f"T{k}" for k in range(system.n_types)]


def write_psf(path: str, system: System) -> None:
    """A PSF of the system (one segment, one residue per molecule; types
    T0, T1, ... of ``type_names``), for the reference's own readers."""
    names = type_names(system)
    q = system.scaled_charge / SQRT_COULOMB_CONSTANT
    with open(path, "w") as fh:
        fh.write("PSF\n\n       1 !NTITLE\n REMARKS synthetic system\n\n")
        fh.write(f"{system.n_atoms:8d} !NATOM\n")
        for i in range(system.n_atoms):
            fh.write(f"{i + 1:8d} SYS  {int(system.molecule[i]) + 1:<5d}MOL  A{i + 1:<4d} "
                     f"{names[system.atom_type[i]]:<6s}{float(q[i])!r:>24s} {float(system.mass[i])!r:>20s}           0\n")
        for key, recs, per_line in (("!NBOND: bonds", system.bonds, 4), ("!NTHETA: angles", system.angles, 3),
                                    ("!NPHI: dihedrals", system.dihedrals, 2), ("!NIMPHI: impropers", [], 2)):
            fh.write(f"\n{len(recs):8d} {key}\n")
            for k in range(0, len(recs), per_line):
                fh.write("".join(f"{a + 1:8d}" for rec in recs[k:k + per_line] for a in rec) + "\n")


def write_par(path: str, system: System) -> None:
    names = type_names(system)
    with open(path, "w") as fh:
        fh.write("* synthetic parameters\n*\n\nNONBONDED nbxmod 5 atom cdiel shift vatom vdistance vswitch -\n"
                 "cutnb 14.0 ctofnb 12.0 ctonnb 10.0 eps 1.0 e14fac 1.0 wmin 1.5\n")
        for k, (eps, rmin, eps14, rmin14) in enumerate(system.type_params):
            fh.write(f"{names[k]:<8s} 0.0 {-float(eps)!r} {float(rmin)!r} 0.0 {-float(eps14)!r} {float(rmin14)!r}\n")
        combined = systems.lj_table_from_types(system.type_params)
        fixes = [(i, j) for i in range(system.n_types) for j in range(i, system.n_types)
                 if not np.array_equal(combined[i, j], system.lj_table[i, j])]
        if fixes:                    # table entries the combination rule does not give
            fh.write("\nNBFIX\n")
            for i, j in fixes:
                fh.write(f"{names[i]:<8s} {names[j]:<8s} " + " ".join(repr(float(v)) for v in system.lj_table[i, j])
                         + "\n")
        fh.write("\nEND\n")


def write_xyz(path: str, system: System) -> None:
    with open(path, "w") as fh:
        fh.write(f"{system.n_atoms}\n{system.name}\n")
        for i, (x, y, z) in enumerate(system.positions):
            fh.write(f"A{i + 1} {float(x)!r} {float(y)!r} {float(z)!r}\n")
