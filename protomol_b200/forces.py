"""Host-side mirror of ProtoMol's force interface for the nonbonded path.

The classes here mirror what a ProtoMol user sees:

* :class:`Topology` -- ``Topology<PeriodicBoundaryConditions,
  CubicCellManager>`` (``topology/Topology.h``): atoms, exclusions, the
  Lennard-Jones table, coulombScalingFactor, box and cell size;
* :class:`ForceFactory` -- ``ForceFactory::make`` (``frontend/ForceFactoryDetails.cpp:48-293``):
  a force definition string such as
  ``"LennardJones CoulombEwaldReal -algorithm NonbondedCutoff -switchingFunction C2
  -switchingFunction Cutoff -switchon 10 -cutoff 12 -alpha 0.32 -cutoff 12 -cutoff 12"``
  or ``"Coulomb -algorithm PMEwald -reciprocal -correction -interpolation BSpline
  -gridsize 64 64 64 -cutoff 12 -alpha 0.32"`` becomes a force object;
* :class:`SystemForce` -- ``SystemForce::evaluate(topo, positions, forces,
  energies)`` (``forces/SystemForce.h:18-76``): forces and energies are
  accumulated (+=) into the caller's arrays.

Every evaluation runs on the GPU through libpmgpu.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check

_VP = C.c_void_p


class ScalarStructure:
    """The slots of ``ScalarStructure`` (``base/ScalarStructure.h:25-54``)
    this path writes, with the ``virial()`` and ``molecularVirial()``
    switches.  The molecular virial needs the molecule positions
    (:meth:`Topology.set_molecule_positions`)."""

    def __init__(self, virial: bool = True, molecular_virial: bool = False):
        self.lennard_jones = 0.0
        self.coulomb = 0.0
        self.virial_tensor = np.zeros(9)
        self.molecular_virial_tensor = np.zeros(9)
        self.virial = virial
        self.molecular_virial = molecular_virial

    def clear(self):
        self.lennard_jones = 0.0
        self.coulomb = 0.0
        self.virial_tensor[:] = 0.0
        self.molecular_virial_tensor[:] = 0.0

    def potential_energy(self) -> float:
        return self.lennard_jones + self.coulomb


class Topology:
    """A pmgpu_system built from a :class:`protomol_b200.systems.System`."""

    def __init__(self, system, device: int = 0):
        lib = _lib.load()
        h = _VP()
        check(lib.pmgpu_system_create(device, C.byref(h)))
        self.handle = h
        self.system = system
        self.n_atoms = system.n_atoms
        self._forces = weakref.WeakSet()
        self.set_topology(system)
        if getattr(system, "periodic", True):   # a vacuum system needs no box
            self.set_box(system.box, system.cell_size)

    def set_topology(self, s):
        lib = _lib.load()
        q = np.ascontiguousarray(s.scaled_charge, np.float64)
        ty = np.ascontiguousarray(s.atom_type, np.int32)
        mol = np.ascontiguousarray(s.molecule, np.int32)
        lj = np.ascontiguousarray(s.lj_table, np.float64)
        ex = np.ascontiguousarray(s.exclusions[:, :2], np.int32)
        cl = np.ascontiguousarray(s.exclusions[:, 2], np.int32)
        ck = np.ascontiguousarray(s.exclusion_check, np.int32)
        p = lambda a: a.ctypes.data_as(_VP) if a.size else None
        check(lib.pmgpu_set_topology(self.handle, s.n_atoms, p(q), p(ty), p(mol), s.n_types, p(lj),
                                     int(ex.shape[0]), p(ex), p(cl), p(ck), float(s.csf)), self.handle)
        self.n_atoms = s.n_atoms
        self.n_types = s.n_types

    def set_box(self, box, cell_size):
        lib = _lib.load()
        b = np.ascontiguousarray(box, np.float64).reshape(4, 3)
        arr = [(C.c_double * 3)(*b[k]) for k in range(4)]
        check(lib.pmgpu_set_box(self.handle, *arr, float(cell_size)), self.handle)

    @property
    def stream(self) -> int:
        return _lib.load().pmgpu_stream(self.handle) or 0

    def launch_count(self) -> int:
        return int(_lib.load().pmgpu_launch_count(self.handle))

    @property
    def tuning(self) -> dict:
        """The launch shapes of this system's evaluations (pmgpu_get_tuning)."""
        t = _lib.Tuning()
        check(_lib.load().pmgpu_get_tuning(self.handle, C.byref(t)), self.handle)
        return t.as_dict()

    def set_tuning(self, **kw):
        """pmgpu_set_tuning with the given fields changed."""
        t = _lib.Tuning()
        lib = _lib.load()
        check(lib.pmgpu_get_tuning(self.handle, C.byref(t)), self.handle)
        for k, v in kw.items():
            setattr(t, k, v)
        check(lib.pmgpu_set_tuning(self.handle, C.byref(t)), self.handle)

    def autotune(self, forces, positions, evals: int = 5, virial: bool = True) -> dict:
        """pmgpu_autotune: times candidate launch shapes on these forces and
        positions and keeps the fastest; returns it with its ms per evaluation."""
        lib = _lib.load()
        pos = np.ascontiguousarray(positions, np.float64)
        arr = (_VP * len(forces))(*[f.handle for f in forces])
        t = _lib.Tuning()
        check(lib.pmgpu_autotune(self.handle, len(forces), arr, pos.ctypes.data_as(_VP),
                                 _lib.FLAG_VIRIAL if virial else 0, int(evals), C.byref(t)), self.handle)
        return t.as_dict()

    def set_molecule_positions(self, positions):
        """pmgpu_set_molecule_positions: ``GenericTopology::molecules[m].
        position`` for every molecule (n_molecules, 3), the points the
        molecular virial measures from (ProtoMol sets them with
        buildMolecularCenterOfMass or minimalImage)."""
        p = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
        check(_lib.load().pmgpu_set_molecule_positions(self.handle, p.shape[0], p.ctypes.data_as(_VP)),
              self.handle)

    def set_pair_list(self, skin: float, rebuild_every: int):
        """pmgpu_set_pair_list: keep the column layout's pair list, built with
        the cutoff plus ``skin`` A, for ``rebuild_every`` evaluations."""
        check(_lib.load().pmgpu_set_pair_list(self.handle, float(skin), int(rebuild_every)), self.handle)

    def pair_list_builds(self) -> int:
        return int(_lib.load().pmgpu_pair_list_builds(self.handle))

    def pair_layout(self) -> str:
        """Cluster layout of the last evaluation's mixed cutoff forces:
        'columns' (fixed-point coordinates in z-sorted columns), 'cells'
        (clusters inside the reference cells), 'fp64' (the FP64 pair
        kernels, tuning fp64_pairs) or '' (none yet)."""
        return {1: "cells", 2: "columns", 3: "fp64"}.get(int(_lib.load().pmgpu_pair_layout(self.handle)), "")

    def cells(self):
        cells = np.zeros((self.n_atoms, 3), np.int32)
        dims = np.zeros(3, np.int32)
        check(_lib.load().pmgpu_get_cells(self.handle, cells.ctypes.data_as(_VP), dims.ctypes.data_as(_VP)),
              self.handle)
        return cells, tuple(int(d) for d in dims)

    def close(self):
        """Destroys the forces made on this topology, then the system (the
        C side frees a force's buffers through its system)."""
        if getattr(self, "handle", None):
            for f in list(getattr(self, "_forces", ())):
                f.close()
            _lib.load().pmgpu_system_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SystemForce:
    """One GPU force object (a pmgpu_force)."""

    keyword = ""

    def __init__(self, topo: Topology, handle, ident: str, params):
        self.topo = topo
        self.handle = handle
        self.id = ident
        self.params = params
        topo._forces.add(self)

    def getKeyword(self) -> str:  # noqa: N802 (mirrors Force::getKeyword)
        return self.keyword

    def getIdNoAlias(self) -> str:  # noqa: N802
        return self.id

    def evaluate(self, topo: Topology, positions: np.ndarray, forces: np.ndarray,
                 energies: ScalarStructure):
        evaluate_group(topo, [self], positions, forces, energies)

    def close(self):
        # only while the owning system is alive: Topology.close() closes its
        # forces first, so a force collected after its topology is a no-op
        if getattr(self, "handle", None) and getattr(self.topo, "handle", None):
            _lib.load().pmgpu_force_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pairs(self, positions, cap=None):
        """Within-cutoff pair set of this force on ``positions`` (diagnostic; for
        PMEwald -real the pairs of its real-space term)."""
        pos = np.ascontiguousarray(positions, np.float64)
        cap = cap or max(1024, pos.shape[0] * 1200)
        out = np.zeros((cap, 2), np.int32)
        cnt = C.c_longlong(0)
        lib = _lib.load()
        for attempt in range(3):
            # a list that outgrew its estimate is grown and the recording rerun
            rc = lib.pmgpu_get_pairs(self.topo.handle, self.handle, pos.ctypes.data_as(_VP), C.byref(cnt),
                                     out.ctypes.data_as(_VP), cap)
            if rc != 7 or cnt.value > cap:
                break
        check(rc, self.topo.handle)
        return out[: cnt.value]


class NonbondedCutoffSystemForce(SystemForce):
    keyword = "NonbondedCutoff"


class NonbondedSimpleFullSystemForce(SystemForce):
    keyword = "NonbondedSimpleFull"


class NonbondedPMEwaldSystemForce(SystemForce):
    keyword = "PMEwald"

    @property
    def alpha(self) -> float:
        a = C.c_double(0.0)
        check(_lib.load().pmgpu_pme_alpha(self.handle, C.byref(a)))
        return a.value


def molecular_centers(molecule, positions, mass=None) -> np.ndarray:
    """buildMolecularCenterOfMass (topology/topologyutilities.cpp:761-769):
    the centre of mass of every molecule, its atoms taken in index order and
    Kahan-summed as molecularCenterOfMass (:729-759) does, unit masses unless
    ``mass`` is given.  Returns (max molecule id + 1, 3); the positions for
    :meth:`Topology.set_molecule_positions`."""
    mol = np.asarray(molecule, np.int64)
    pos = np.asarray(positions, np.float64).reshape(-1, 3)
    m = np.ones(mol.shape[0]) if mass is None else np.asarray(mass, np.float64)
    nm = int(mol.max()) + 1 if mol.size else 0
    order = np.argsort(mol, kind="stable")             # each molecule's atoms in index order
    counts = np.bincount(mol, minlength=nm)
    first = np.concatenate([[0], np.cumsum(counts)[:-1]])
    rank = np.empty(mol.shape[0], np.int64)
    rank[order] = np.arange(mol.shape[0]) - first[mol[order]]
    center = np.zeros((nm, 3))
    comp = np.zeros((nm, 3))
    total = np.zeros(nm)
    by_rank = np.argsort(rank, kind="stable")
    bounds = np.searchsorted(rank[by_rank], np.arange(int(counts.max(initial=0)) + 1))
    for r in range(len(bounds) - 1):
        sel = by_rank[bounds[r]:bounds[r + 1]]
        ids = mol[sel]
        x = pos[sel] * m[sel, None]
        if r == 0:
            center[ids] = x
            total[ids] = m[sel]
            continue
        total[ids] += m[sel]
        y = x - comp[ids]
        t = center[ids] + y
        comp[ids] = (t - center[ids]) - y
        center[ids] = t
    with np.errstate(invalid="ignore", divide="ignore"):
        out = center / total[:, None]
    out[counts == 0] = 0.0
    return out


def evaluate_group(topo: Topology, forces, positions, force_accum, energies: ScalarStructure):
    """ForceGroup::evaluateSystemForces (forces/ForceGroup.cpp:43-96) for GPU
    forces: one host->device copy, all forces, one device->host copy."""
    lib = _lib.load()
    pos = np.ascontiguousarray(positions, np.float64)
    if force_accum.dtype != np.float64 or not force_accum.flags.c_contiguous:
        raise ValueError("forces must be a C-contiguous float64 (N, 3) array")
    if pos.shape != (topo.n_atoms, 3) or force_accum.shape != (topo.n_atoms, 3):
        raise ValueError("positions / forces must have shape (N, 3)")
    arr = (_VP * len(forces))(*[f.handle for f in forces])
    mol = getattr(energies, "molecular_virial", False)
    e = _lib.EnergiesMol() if mol else _lib.Energies()
    flags = (_lib.FLAG_VIRIAL if energies.virial else 0) | (_lib.FLAG_MOLECULAR_VIRIAL if mol else 0)
    check(lib.pmgpu_evaluate(topo.handle, len(forces), arr, pos.ctypes.data_as(_VP),
                             force_accum.ctypes.data_as(_VP), C.byref(e), flags), topo.handle)
    energies.lennard_jones += e.lennard_jones
    energies.coulomb += e.coulomb
    # with the molecular virial alone, the atomic slots still receive the
    # pairs of different molecules (ScalarStructure::addVirial(f, d, comDiff))
    if energies.virial or mol:
        energies.virial_tensor += np.array(list(e.virial))
    if mol:
        energies.molecular_virial_tensor += np.array(list(e.molecular_virial))


def adjoint(topo: Topology, forces, positions, v=None):
    """Backward pass of ``evaluate_group`` (pmgpu_adjoint): gradients of the
    forces' total energy w.r.t. the scaled charges (N) and the LJ table
    (T x T x 4, {A, B, A14, B14}), and with ``v`` (N x 3) the Hessian-vector
    product of the pair terms.  Returns a dict of numpy arrays."""
    lib = _lib.load()
    pos = np.ascontiguousarray(positions, np.float64)
    n, t = topo.n_atoms, topo.n_types
    dq = np.zeros(n)
    dlj = np.zeros((t, t, 4))
    en = np.zeros(2)
    hv = None
    vv = None
    if v is not None:
        vv = np.ascontiguousarray(v, np.float64)
        hv = np.zeros((n, 3))
    arr = (_VP * len(forces))(*[f.handle for f in forces])
    check(lib.pmgpu_adjoint(topo.handle, len(forces), arr, pos.ctypes.data_as(_VP),
                            vv.ctypes.data_as(_VP) if vv is not None else None, dq.ctypes.data_as(_VP),
                            dlj.ctypes.data_as(_VP), hv.ctypes.data_as(_VP) if hv is not None else None,
                            en.ctypes.data_as(_VP)), topo.handle)
    return {"dE_dq": dq, "dE_dlj": dlj, "hv": hv, "lennard_jones": en[0], "coulomb": en[1]}


def hessian(topo: Topology, forces, positions) -> np.ndarray:
    """pmgpu_hessian: the dense 3N x 3N Hessian of the forces' pair terms
    (Hessian::evaluate's blocks, integrators/Hessian.cpp:456-623)."""
    lib = _lib.load()
    pos = np.ascontiguousarray(positions, np.float64)
    n3 = 3 * topo.n_atoms
    h = np.zeros((n3, n3))
    arr = (_VP * len(forces))(*[f.handle for f in forces])
    check(lib.pmgpu_hessian(topo.handle, len(forces), arr, pos.ctypes.data_as(_VP), h.ctypes.data_as(_VP)),
          topo.handle)
    return h


def lj_parameter_gradient(type_params, dE_dlj):
    """Chain rule from the LJ-table gradient of ``adjoint`` to the per-type
    parameters of the PAR file: returns (T, 4) = dE/d(eps, Rmin/2, eps14,
    Rmin14/2), the table being built by the CHARMM combination rule
    (frontend/buildTopology.cpp:646-664): A = (R_x + R_y)^12 sqrt(e_x e_y),
    B = 2 (R_x + R_y)^6 sqrt(e_x e_y), likewise A14 / B14."""
    tp = np.asarray(type_params, np.float64)
    g = np.asarray(dE_dlj, np.float64)
    out = np.zeros_like(tp)
    for k, (ie, ir) in enumerate(((0, 1), (2, 3))):
        eps, rh = tp[:, ie], tp[:, ir]
        r = rh[:, None] + rh[None, :]
        e = np.sqrt(eps[:, None] * eps[None, :])
        A = r ** 12 * e
        B = 2.0 * r ** 6 * e
        gA, gB = g[:, :, 2 * k], g[:, :, 2 * k + 1]
        m = gA * A + gB * B                  # d/d ln(e): both entries scale with sqrt(e_x e_y)
        with np.errstate(divide="ignore", invalid="ignore"):   # undefined (nan) where eps = 0
            out[:, ie] = (m.sum(1) + m.sum(0)) / (2.0 * eps)
        nr = (12.0 * gA * A + 6.0 * gB * B) / r
        out[:, ir] = nr.sum(1) + nr.sum(0)
    return out


# --------------------------------------------------------------------------
# keyword parsing
# --------------------------------------------------------------------------
_POTENTIALS = ("LennardJones", "Coulomb", "CoulombEwaldReal",
               "LennardJonesTable", "CoulombTable", "CoulombEwaldRealTable")
_SWITCHES = ("Universal", "Cutoff", "C1", "C2", "Shift")
# Table potentials (forces/*TableForce.h): the switching function is the
# tabulated one and the pair applies Universal.  LennardJonesTable and
# CoulombTable name it in their id; CoulombEwaldRealTable's is Cutoff and
# hidden (CoulombEwaldRealTableForce.h:120-124).
_TABLES = ("LennardJonesTable", "CoulombTable", "CoulombEwaldRealTable")
# (real, reciprocal, correction) of the registered PMEwald exemplars
# (factories/registerForceExemplarsFastElectrostatic.cpp:50-55)
_PME_REGISTERED = ((True, True, True), (True, False, False), (True, False, True),
                   (False, True, False), (False, True, True), (False, False, True))


@dataclass
class _Param:
    keyword: str
    default: object = None


def _switch_params(sw):
    # getParameters() of each switching function
    return {"C2": [_Param("-switchon"), _Param("-cutoff")], "C1": [_Param("-cutoff")],
            "Cutoff": [_Param("-cutoff")], "Shift": [_Param("-cutoff")], "Universal": []}[sw]


def _pot_params(pot):
    return [_Param("-alpha")] if pot in ("CoulombEwaldReal", "CoulombEwaldRealTable") else []


def _term_params(pot, sw):
    """OneAtomPair::getParameters of one term: the potential's parameters,
    then the switching function's.  A table potential's parameters are its
    tabulated switching function's (its cutoff is that function's), then
    -alpha (forces/CoulombEwaldRealTableForce.h:126-131); the pair's Universal
    switch has none."""
    if pot in _TABLES:
        return _switch_params(sw) + _pot_params(pot)
    return _pot_params(pot) + _switch_params(sw)


def _term_values(pot, sw, vals, k):
    """(switchon, cutoff, alpha, next k) from the parsed values of a term."""
    alpha = on = rc = 0.0
    if pot in ("CoulombEwaldReal",):
        alpha = vals[k]; k += 1
    if sw == "C2":
        on, rc = vals[k], vals[k + 1]; k += 2
    elif sw in ("C1", "Cutoff", "Shift"):
        rc = vals[k]; k += 1
    if pot == "CoulombEwaldRealTable":
        alpha = vals[k]; k += 1
    return on, rc, alpha, k


def _assign_switches(names, sws):
    """The -switchingFunction words of an id in term order: every term names
    one except CoulombEwaldRealTable (tabulated Cutoff, hidden); None when the
    count does not match."""
    shown = [n != "CoulombEwaldRealTable" for n in names]
    if sum(shown) != len(sws):
        return None
    it = iter(sws)
    return [next(it) if s else "Cutoff" for s in shown]


def _parse_values(tokens, params):
    """Positional keyword matching of ForceFactoryDetails::doMake
    (frontend/ForceFactoryDetails.cpp:192-249): for each parameter in
    getParameters() order, scan forward for its keyword (wrapping around once)
    and take the next token; an empty keyword takes the token after the
    previous match."""
    values = []
    pos = 0
    found_last = False
    for p in params:
        val = None
        if p.keyword == "":
            if found_last and pos < len(tokens):
                val = tokens[pos]
                pos += 1
        else:
            scanned = 0
            k = pos
            while scanned < len(tokens) + 1:
                if k >= len(tokens):
                    k = 0
                if k < len(tokens) and tokens[k].lower() == p.keyword.lower() and k + 1 < len(tokens):
                    val = tokens[k + 1]
                    pos = k + 2
                    break
                k += 1
                scanned += 1
        found_last = val is not None
        if val is None:
            val = p.default
        values.append(val)
    return values


def parse_definition(definition: str) -> dict:
    """Parses a force definition string into its parameters (no GPU needed).

    Returns ``{"kind": "cut", "terms": [(sw, pot, switchon, cutoff, alpha)],
    "algo_cutoff": rc}`` or ``{"kind": "pme", "real": .., "reciprocal": ..,
    "correction": .., "grid": (nx, ny, nz), "order": P, "cutoff": rc,
    "accuracy": a, "alpha": alpha}``; raises ValueError with the
    reference's kind of message when the definition does not match.
    """
    toks = definition.split()
    if toks and toks[0].lower() == "force":
        toks = toks[1:]
    # the factory compares keywords, policies and values without case
    # (frontend/ForceFactoryDetails.cpp:68-122, ltstrNocase / equalNocase)
    canon = {w.lower(): w for w in _POTENTIALS + _SWITCHES +
             ("NonbondedCutoff", "NonbondedSimpleFull", "PMEwald", "BSpline")}
    names, sws, algorithm, interp, flags, rest = [], [], None, None, set(), []
    i = 0
    while i < len(toks):
        t = toks[i]
        tl = t.lower()
        nxt = canon.get(toks[i + 1].lower(), toks[i + 1]) if i + 1 < len(toks) else None
        if canon.get(tl) in _POTENTIALS:
            names.append(canon[tl])
        elif tl == "-switchingfunction" and nxt is not None:
            sws.append(nxt); i += 1
        elif tl == "-algorithm" and nxt is not None:
            algorithm = nxt; i += 1
        elif tl == "-interpolation" and nxt is not None:
            interp = nxt; i += 1
        elif tl in ("-real", "-reciprocal", "-correction"):
            flags.add(tl[1:])
        else:
            rest.append(t)
        i += 1
    if algorithm == "NonbondedCutoff":
        term_sws = _assign_switches(names, sws) if 1 <= len(names) <= 2 else None
        if term_sws is None or any(s not in _SWITCHES for s in term_sws):
            raise ValueError(f"Could not find a complete match for '{definition}'")
        params = []
        for n, s in zip(names, term_sws):
            # OneAtomPair[Two]::getParameters order: force1, switch1, force2, switch2
            params += _term_params(n, s)
        params.append(_Param("-cutoff"))
        vals = _parse_values(rest, params)
        if any(v is None for v in vals):
            raise ValueError(f"force {definition}: missing parameter(s)")
        vals = [float(v) for v in vals]
        terms, k = [], 0
        for n, s in zip(names, term_sws):
            on, rc, alpha, k = _term_values(n, s, vals, k)
            terms.append((s, n, on, rc, alpha))
        return {"kind": "cut", "terms": terms, "algo_cutoff": vals[k]}
    if algorithm == "NonbondedSimpleFull":
        # vacuum all pairs; a Universal switch is not written in the id, so
        # either every term names its switch or none does
        if any(n in _TABLES for n in names) or not 1 <= len(names) <= 2 or (sws and len(sws) != len(names)) or any(s not in _SWITCHES for s in sws):
            raise ValueError(f"Could not find a complete match for '{definition}'")
        sws = sws or ["Universal"] * len(names)
        params = []
        for n, s in zip(names, sws):
            params += _pot_params(n) + _switch_params(s)
        params.append(_Param("-blocksize", 32))
        vals = _parse_values(rest, params)
        if any(v is None for v in vals):
            raise ValueError(f"force {definition}: missing parameter(s)")
        vals = [float(v) for v in vals]
        terms, k = [], 0
        for n, s in zip(names, sws):
            alpha = on = rc = 0.0
            if n == "CoulombEwaldReal":
                alpha = vals[k]; k += 1
            if s == "C2":
                on, rc = vals[k], vals[k + 1]; k += 2
            elif s in ("C1", "Cutoff", "Shift"):
                rc = vals[k]; k += 1
            terms.append((s, n, on, rc, alpha))
        return {"kind": "full", "terms": terms}
    if algorithm == "PMEwald":
        # the registered exemplars (factories/registerForceExemplarsFastElectrostatic.cpp:50-55)
        # all take the Cutoff switch, which their id leaves unwritten, and
        # exist for these (real, reciprocal, correction) sets only
        terms_on = ("real" in flags, "reciprocal" in flags, "correction" in flags)
        if (names != ["Coulomb"] or (interp or "BSpline") != "BSpline" or sws not in ([], ["Cutoff"])
                or terms_on not in _PME_REGISTERED):
            raise ValueError(f"Could not find a complete match for '{definition}'")
        params = [_Param("-gridsize"), _Param(""), _Param(""), _Param("-cutoff"),
                  _Param("-order", 4), _Param("-accuracy", 1e-6), _Param("-alpha", -1.0)]
        vals = _parse_values(rest, params)
        if any(v is None for v in vals):
            raise ValueError(f"force {definition}: missing parameter(s)")
        return {"kind": "pme", "real": int("real" in flags), "reciprocal": int("reciprocal" in flags),
                "correction": int("correction" in flags), "grid": tuple(int(v) for v in vals[:3]),
                "cutoff": float(vals[3]), "order": int(vals[4]), "accuracy": float(vals[5]),
                "alpha": float(vals[6])}
    raise ValueError(f"Could not find a complete match for '{definition}'")


def cutoff_ident(terms) -> str:
    """getIdNoAlias of a NonbondedCutoffSystemForce: OneAtomPair[Two]::getId
    (forces/OneAtomPairTwo.h:97-106) -- the potentials' keywords, their own
    (tabulated) switching functions, then the pair's switching functions
    (Universal is not written) -- and the algorithm."""
    heads = " ".join(t[1] for t in terms)
    tails = "".join(f" -switchingFunction {t[0]}" for t in terms
                    if t[1] in ("LennardJonesTable", "CoulombTable"))
    outer = "".join(f" -switchingFunction {t[0]}" for t in terms if t[1] not in _TABLES)
    return heads + tails + outer + " -algorithm NonbondedCutoff"


class ForceFactory:
    """``ForceFactory::make`` for the GPU nonbonded forces."""

    @staticmethod
    def make(topo: Topology, definition: str, precision: str = "mixed") -> SystemForce:
        lib = _lib.load()
        spec = parse_definition(definition)
        prec = _lib.PRECISION[precision]
        h = _VP()
        if spec["kind"] == "cut":
            cp = _lib.CutoffParams()
            cp.n_terms = len(spec["terms"])
            for t, (s, n, on, rc, alpha) in enumerate(spec["terms"]):
                cp.pot[t] = _lib.POT[n]
                cp.sw[t] = _lib.SW[s]
                cp.switchon[t] = on
                cp.cutoff[t] = rc
                cp.alpha[t] = alpha
            cp.algorithm_cutoff = spec["algo_cutoff"]
            cp.precision = prec
            check(lib.pmgpu_cutoff_create(topo.handle, C.byref(cp), C.byref(h)), topo.handle)
            return NonbondedCutoffSystemForce(topo, h, cutoff_ident(spec["terms"]), spec)
        if spec["kind"] == "full":
            cp = _lib.CutoffParams()
            cp.n_terms = len(spec["terms"])
            for t, (s, n, on, rc, alpha) in enumerate(spec["terms"]):
                cp.pot[t] = _lib.POT[n]
                cp.sw[t] = _lib.SW[s]
                cp.switchon[t] = on
                cp.cutoff[t] = rc
                cp.alpha[t] = alpha
            cp.precision = prec
            check(lib.pmgpu_full_create(topo.handle, C.byref(cp), C.byref(h)), topo.handle)
            ident = (" ".join(t[1] for t in spec["terms"]) +
                     "".join(f" -switchingFunction {t[0]}" for t in spec["terms"] if t[0] != "Universal") +
                     " -algorithm NonbondedSimpleFull")
            return NonbondedSimpleFullSystemForce(topo, h, ident, spec)
        pp = _lib.PmeParams()
        pp.real, pp.reciprocal, pp.correction = spec["real"], spec["reciprocal"], spec["correction"]
        for k in range(3):
            pp.grid[k] = spec["grid"][k]
        pp.cutoff, pp.order, pp.accuracy, pp.alpha = spec["cutoff"], spec["order"], spec["accuracy"], spec["alpha"]
        pp.precision = prec
        check(lib.pmgpu_pme_create(topo.handle, C.byref(pp), C.byref(h)), topo.handle)
        ident = ("Coulomb -algorithm PMEwald" + "".join(f" -{f}" for f in ("real", "reciprocal", "correction")
                                                       if spec[f]) + " -interpolation BSpline")
        return NonbondedPMEwaldSystemForce(topo, h, ident, spec)
