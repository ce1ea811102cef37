"""Python access to the parity oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke``
and by ``bench.py``'s CPU-baseline leg, never by the product package.

Two oracles live here:

* ``liboracle`` -- the C restatement in ``oracle/pmoracle.c`` (built into
  ``oracle/_build/libpmoracle.so`` by :func:`build`), called through ctypes;
* ``run_reference`` -- the reference's own force classes compiled from the
  ProtoMol sources (``oracle/ref/Makefile`` -> ``oracle/_ref/pmref``), run as a
  subprocess on a system file.  It exists only where it was built.

Force specifications are plain dicts shared by both:

``{"kind": "cut", "terms": [(sw, pot, switchon, cutoff, alpha), ...],
"algo_cutoff": rc}``, ``{"kind": "pme", "real": 0, "reciprocal": 1,
"correction": 1, "grid": (nx, ny, nz), "order": 4, "cutoff": rc,
"accuracy": 1e-6, "alpha": a}`` and ``{"kind": "full", "terms": [...]}``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(BUILD, "libpmoracle.so")

SW = {"Universal": 0, "Cutoff": 1, "C1": 2, "C2": 3, "Shift": 4}
POT = {"LennardJones": 1, "Coulomb": 2, "CoulombEwaldReal": 3,
       "LennardJonesTable": 4, "CoulombTable": 5, "CoulombEwaldRealTable": 6}


def build(force: bool = False) -> str:
    """Compile the C restatement (plain gcc, no FMA contraction)."""
    src = os.path.join(HERE, "pmoracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "pmoracle.h"))):
        os.makedirs(BUILD, exist_ok=True)
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared",
                               "-o", LIB, src, "-lm"])
    return LIB


class _System(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int), ("pos", C.c_void_p), ("q", C.c_void_p),
        ("type", C.c_void_p), ("mol", C.c_void_p), ("n_types", C.c_int),
        ("lj", C.c_void_p), ("n_excl", C.c_int), ("excl", C.c_void_p),
        ("excl_check", C.c_void_p), ("box", C.c_double * 12), ("csf", C.c_double),
        ("cell_size", C.c_double), ("mol_pos", C.c_void_p), ("no_virial", C.c_int),
    ]


class _Cut(C.Structure):
    _fields_ = [
        ("n_terms", C.c_int), ("pot", C.c_int * 2), ("sw", C.c_int * 2),
        ("switchon", C.c_double * 2), ("sw_cutoff", C.c_double * 2),
        ("alpha", C.c_double * 2), ("algo_cutoff", C.c_double),
    ]


class _Pme(C.Structure):
    _fields_ = [
        ("real", C.c_int), ("reciprocal", C.c_int), ("correction", C.c_int),
        ("grid", C.c_int * 3), ("order", C.c_int), ("cutoff", C.c_double),
        ("accuracy", C.c_double), ("alpha", C.c_double),
    ]


class _Result(C.Structure):
    _fields_ = [
        ("lennard_jones", C.c_double), ("coulomb", C.c_double),
        ("virial", C.c_double * 9), ("n_pairs", C.c_longlong), ("alpha", C.c_double),
        ("e_real", C.c_double), ("e_recip", C.c_double), ("e_intra", C.c_double),
        ("e_self", C.c_double), ("e_charged", C.c_double), ("out_of_grid", C.c_int),
        ("mol_virial", C.c_double * 9),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.pmo_poly5.restype = C.c_double
        _lib.pmo_poly5.argtypes = [C.c_double]
        _lib.pmo_lookup_table.restype = C.c_longlong
        _lib.pmo_lookup_table.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                          C.c_void_p, C.c_longlong]
    return _lib


def lookup_table(pot, sw, switchon, cutoff, alpha=0.0) -> np.ndarray:
    """The LookUpTableBase table of a table potential (pmo_lookup_table)."""
    p, s = POT[pot] if isinstance(pot, str) else pot, SW[sw] if isinstance(sw, str) else sw
    n = lib().pmo_lookup_table(p, s, switchon, cutoff, alpha, None, 0)
    if n < 0:
        raise ValueError(f"{pot} is not a table potential")
    out = np.zeros(n)
    lib().pmo_lookup_table(p, s, switchon, cutoff, alpha, out.ctypes.data, n)
    return out


class _Keep:
    """Holds the numpy arrays a _System points into."""

    def __init__(self, system, positions=None, mol_pos=None, virial=True):
        pos = system.positions if positions is None else positions
        self.pos = np.ascontiguousarray(pos, np.float64)
        self.q = np.ascontiguousarray(system.scaled_charge, np.float64)
        self.type = np.ascontiguousarray(system.atom_type, np.int32)
        self.mol = np.ascontiguousarray(system.molecule, np.int32)
        self.lj = np.ascontiguousarray(system.lj_table, np.float64)
        self.excl = np.ascontiguousarray(system.exclusions, np.int32)
        self.chk = np.ascontiguousarray(system.exclusion_check, np.int32)
        s = _System()
        s.n_atoms = self.pos.shape[0]
        s.pos = self.pos.ctypes.data
        s.q = self.q.ctypes.data
        s.type = self.type.ctypes.data
        s.mol = self.mol.ctypes.data
        s.n_types = self.lj.shape[0]
        s.lj = self.lj.ctypes.data
        s.n_excl = self.excl.shape[0]
        s.excl = self.excl.ctypes.data if self.excl.size else None
        s.excl_check = self.chk.ctypes.data if self.chk.size else None
        for k, v in enumerate(np.asarray(system.box, np.float64).ravel()):
            s.box[k] = v
        s.csf = system.csf
        s.cell_size = system.cell_size
        if mol_pos is not None:
            self.mol_pos = np.ascontiguousarray(mol_pos, np.float64).reshape(-1, 3)
            if self.mol_pos.shape[0] < int(self.mol.max()) + 1:
                raise ValueError("one position per molecule is needed")
            s.mol_pos = self.mol_pos.ctypes.data
        s.no_virial = 0 if virial else 1
        self.s = s


def _cut_params(spec) -> _Cut:
    p = _Cut()
    terms = spec["terms"]
    p.n_terms = len(terms)
    for k, (sw, pot, on, rc, alpha) in enumerate(terms):
        p.sw[k] = SW[sw] if isinstance(sw, str) else sw
        p.pot[k] = POT[pot] if isinstance(pot, str) else pot
        p.switchon[k] = on
        p.sw_cutoff[k] = rc
        p.alpha[k] = alpha
    p.algo_cutoff = spec.get("algo_cutoff", max(t[3] for t in terms))
    return p


def _pme_params(spec) -> _Pme:
    p = _Pme()
    p.real = int(spec.get("real", 0))
    p.reciprocal = int(spec.get("reciprocal", 1))
    p.correction = int(spec.get("correction", 1))
    for k, g in enumerate(spec["grid"]):
        p.grid[k] = int(g)
    p.order = int(spec.get("order", 4))
    p.cutoff = float(spec["cutoff"])
    p.accuracy = float(spec.get("accuracy", 1e-6))
    p.alpha = float(spec.get("alpha", -1.0))
    return p


def _result_dict(r: _Result, forces):
    return {
        "forces": forces, "lennard_jones": r.lennard_jones, "coulomb": r.coulomb,
        "virial": np.array(list(r.virial)), "n_pairs": int(r.n_pairs), "alpha": r.alpha,
        "e_real": r.e_real, "e_recip": r.e_recip, "e_intra": r.e_intra,
        "e_self": r.e_self, "e_charged": r.e_charged, "out_of_grid": r.out_of_grid,
        "mol_virial": np.array(list(r.mol_virial)),
    }


def evaluate(system, specs, positions=None, want_pairs=False, pair_cap=None, mol_pos=None, virial=True):
    """Evaluates the force specs in order into one force block (like
    ForceGroup::evaluateSystemForces).  Returns a dict.  ``mol_pos`` (one
    position per molecule) turns the molecular virial on; ``virial=False``
    is ScalarStructure::virial() off."""
    keep = _Keep(system, positions, mol_pos, virial)
    n = keep.pos.shape[0]
    forces = np.zeros((n, 3), np.float64)
    r = _Result()
    pairs = None
    L = lib()
    for spec in specs:
        if spec["kind"] == "cut":
            p = _cut_params(spec)
            if want_pairs:
                cap = pair_cap or n * 1200
                pairs = np.zeros((cap, 2), np.int32)
                L.pmo_cutoff_force(C.byref(keep.s), C.byref(p), forces.ctypes.data_as(C.c_void_p),
                                   C.byref(r), pairs.ctypes.data_as(C.c_void_p), C.c_longlong(cap))
                if r.n_pairs > cap:
                    raise RuntimeError("pair capacity too small")
                pairs = pairs[: r.n_pairs]
            else:
                L.pmo_cutoff_force(C.byref(keep.s), C.byref(p), forces.ctypes.data_as(C.c_void_p),
                                   C.byref(r), None, C.c_longlong(0))
        elif spec["kind"] == "pme":
            p = _pme_params(spec)
            rc = L.pmo_pme_force(C.byref(keep.s), C.byref(p), forces.ctypes.data_as(C.c_void_p), C.byref(r))
            if rc != 0:
                raise RuntimeError("PME oracle needs an orthogonal box")
        elif spec["kind"] == "full":
            p = _cut_params(spec)
            L.pmo_simple_full_force(C.byref(keep.s), C.byref(p), forces.ctypes.data_as(C.c_void_p), C.byref(r))
        else:
            raise ValueError(spec["kind"])
    out = _result_dict(r, forces)
    if want_pairs:
        out["pairs"] = pairs
    return out


def molecular_centers(system, positions=None, mass=None):
    """buildMolecularCenterOfMass (topology/topologyutilities.cpp:761-769)
    with unit masses unless ``mass`` is given: (n_molecules, 3)."""
    keep = _Keep(system, positions)
    nm = int(keep.mol.max()) + 1 if keep.mol.size else 0
    out = np.zeros((nm, 3), np.float64)
    m = None if mass is None else np.ascontiguousarray(mass, np.float64)
    lib().pmo_molecular_centers(C.byref(keep.s), None if m is None else m.ctypes.data_as(C.c_void_p),
                                out.ctypes.data_as(C.c_void_p))
    return out


def pair_hessian(system, spec, positions=None):
    """Dense (3N, 3N) Hessian of a cutoff / all-pairs force's pair terms as
    integrators/Hessian.cpp:456-623 assembles it (LennardJones and Coulomb
    under Universal, C1 or C2 switching); all-pairs forces use plain
    differences (vacuum), cutoff forces the minimal image."""
    keep = _Keep(system, positions)
    n3 = 3 * keep.pos.shape[0]
    H = np.zeros((n3, n3), np.float64)
    p = _cut_params(spec)
    rc = lib().pmo_pair_hessian(C.byref(keep.s), C.byref(p), 1 if spec["kind"] == "full" else 0,
                                H.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise ValueError("no Hessian block for these terms (Hessian.cpp: LJ / Coulomb, Universal / C1 / C2)")
    return H


def cell_assign(system, positions=None):
    keep = _Keep(system, positions)
    cells = np.zeros((keep.pos.shape[0], 3), np.int32)
    dims = np.zeros(3, np.int32)
    oog = lib().pmo_cell_assign(C.byref(keep.s), cells.ctypes.data_as(C.c_void_p),
                                dims.ctypes.data_as(C.c_void_p))
    return cells, tuple(int(d) for d in dims), oog


def fft3d(data: np.ndarray, sign: int) -> np.ndarray:
    a = np.ascontiguousarray(data, np.complex128).copy()
    nx, ny, nz = a.shape
    lib().pmo_fft3d(a.ctypes.data_as(C.c_void_p), nx, ny, nz, sign)
    return a


def poly5(x: float) -> float:
    return lib().pmo_poly5(float(x))


# --------------------------------------------------------------- reference
def run_reference_parallel(system, specs, repeat: int, procs: int, fast: bool = True, timeout=None):
    """``procs`` independent processes of the compiled reference, all running
    at once, each timing ``repeat`` evaluations of the same system (the
    reference's force path is single-threaded: one evaluation uses one core,
    so the host's cores are used by replicas).  Returns the per-process
    seconds per evaluation; the host's throughput is the sum of the rates."""
    exe = os.path.join(REF_DIR, "pmref_fast" if fast else "pmref")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory() as td:
        sp = os.path.join(td, "sys.bin")
        system.save(sp)
        extra = []
        for spec in specs:
            extra += _spec_args(spec)
        outs = [os.path.join(td, f"out{k}.bin") for k in range(procs)]
        ps = [subprocess.Popen([exe, sp, o, str(int(repeat))] + extra, stdout=subprocess.DEVNULL)
              for o in outs]
        try:
            for p in ps:
                if p.wait(timeout=timeout) != 0:
                    raise RuntimeError(f"reference process exited with {p.returncode}")
        finally:
            for p in ps:
                if p.poll() is None:
                    p.kill()
                    p.wait()
        return [float(np.frombuffer(open(o, "rb").read(13 * 8), np.float64)[11]) for o in outs]


def reference_available(fast: bool = False) -> bool:
    return os.path.exists(os.path.join(REF_DIR, "pmref_fast" if fast else "pmref"))


def build_reference(ref_root: str) -> bool:
    """Compile the reference's own sources (only where they are present) and
    record where they came from (``reference_root``)."""
    if not os.path.isdir(os.path.join(ref_root, "framework")):
        return reference_available()
    subprocess.check_call(["make", "-C", os.path.join(HERE, "ref"), f"REF={ref_root}",
                           "-j", str(os.cpu_count() or 4), "-s"])
    with open(os.path.join(REF_DIR, "REFERENCE_ROOT"), "w") as fh:
        fh.write(os.path.abspath(ref_root) + "\n")
    return True


def reference_root():
    """The ProtoMol source tree: $PROTOMOL_REFERENCE, else the tree the
    compiled reference was built from; None when neither is known."""
    env = os.environ.get("PROTOMOL_REFERENCE")
    if env:
        return env
    try:
        with open(os.path.join(REF_DIR, "REFERENCE_ROOT")) as fh:
            return fh.read().strip() or None
    except OSError:
        return None


def _spec_args(spec):
    if spec["kind"] in ("cut", "full"):
        args = [spec["kind"], str(len(spec["terms"]))]
        for sw, pot, on, rc, alpha in spec["terms"]:
            args += [str(SW[sw] if isinstance(sw, str) else sw),
                     str(POT[pot] if isinstance(pot, str) else pot),
                     repr(float(on)), repr(float(rc)), repr(float(alpha))]
        if spec["kind"] == "cut":
            args.append(repr(float(spec.get("algo_cutoff", max(t[3] for t in spec["terms"])))))
        return args
    g = spec["grid"]
    return ["pme", str(int(spec.get("real", 0))), str(int(spec.get("reciprocal", 1))),
            str(int(spec.get("correction", 1))), str(g[0]), str(g[1]), str(g[2]),
            str(int(spec.get("order", 4))), repr(float(spec["cutoff"])),
            repr(float(spec.get("accuracy", 1e-6))), repr(float(spec.get("alpha", -1.0)))]


def run_reference(system, specs, repeat: int = 1, fast: bool = False, timeout=None,
                  molecular_virial=False, virial=True):
    """Runs the compiled reference; returns the same dict as :func:`evaluate`
    plus ``cells``/``dims`` and ``seconds_per_eval`` (when repeat > 1).  With
    ``molecular_virial`` the reference sets the molecule positions itself
    (buildMolecularCenterOfMass, unit masses) and the dict adds
    ``mol_pos`` and ``mol_virial``."""
    exe = os.path.join(REF_DIR, "pmref_fast" if fast else "pmref")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory() as td:
        sp = os.path.join(td, "sys.bin")
        op = os.path.join(td, "out.bin")
        system.save(sp)
        args = [exe, sp, op, str(int(repeat))]
        for spec in specs:
            args += _spec_args(spec)
        env = dict(os.environ, PMREF_MOLVIR="1" if molecular_virial else "0",
                   PMREF_NO_VIRIAL="0" if virial else "1")
        subprocess.run(args, check=True, timeout=timeout, stdout=subprocess.DEVNULL, env=env)
        raw = open(op, "rb").read()
    n = system.n_atoms
    hdr = np.frombuffer(raw[: 13 * 8], np.float64)
    off = 13 * 8
    forces = np.frombuffer(raw[off: off + 24 * n], np.float64).reshape(n, 3).copy()
    off += 24 * n
    dims = tuple(int(x) for x in np.frombuffer(raw[off: off + 12], np.int32))
    off += 12
    cells = np.frombuffer(raw[off: off + 12 * n], np.int32).reshape(n, 3).copy()
    off += 12 * n
    out = {
        "forces": forces, "lennard_jones": float(hdr[0]), "coulomb": float(hdr[1]),
        "virial": hdr[2:11].copy(), "seconds_per_eval": float(hdr[11]),
        "cells": cells, "dims": dims,
    }
    if molecular_virial:
        nm = int(np.frombuffer(raw[off: off + 4], np.int32)[0])
        off += 4
        out["mol_pos"] = np.frombuffer(raw[off: off + 24 * nm], np.float64).reshape(nm, 3).copy()
        off += 24 * nm
        out["mol_virial"] = np.frombuffer(raw[off: off + 72], np.float64).copy()
    return out


def run_reference_hessian(system, specs, timeout=None):
    """ProtoMol's own Hessian (integrators/Hessian.cpp: ``findForces`` over
    a ForceGroup of the given forces, then ``evaluate`` without mass
    re-weighting) on a vacuum system, run by the compiled reference: the
    dense (3N, 3N) matrix.  Its nonbonded part reads separate LennardJones
    and Coulomb forces (one term per spec)."""
    exe = os.path.join(REF_DIR, "pmref")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory() as td:
        sp = os.path.join(td, "sys.bin")
        op = os.path.join(td, "out.bin")
        hp = os.path.join(td, "hess.bin")
        system.save(sp)
        args = [exe, sp, op, "1"]
        for spec in specs:
            args += _spec_args(spec)
        env = dict(os.environ, PMREF_HESSIAN=hp)
        subprocess.run(args, check=True, timeout=timeout, stdout=subprocess.DEVNULL, env=env)
        n3 = 3 * system.n_atoms
        return np.frombuffer(open(hp, "rb").read(), np.float64).reshape(n3, n3).copy()


# ---------------------------------------------------------------- integration
INV_TIMEFACTOR = 0.02045482828087295          # Constant::INV_TIMEFACTOR (base/pmconstants.cpp:49)


TIMEFACTOR = 48.88821290839616      # Constant::TIMEFACTOR (base/pmconstants.cpp:48)


def _shake(c, pos, vel, last, dt):
    a = np.ascontiguousarray(c["atoms"], np.int32)
    r = np.ascontiguousarray(c["rest"], np.float64)
    m = np.ascontiguousarray(c["mass"], np.float64)
    eps, it = c["shake"]
    return lib().pmo_shake(len(r), a.ctypes.data_as(C.c_void_p), r.ctypes.data_as(C.c_void_p),
                           m.ctypes.data_as(C.c_void_p), pos.shape[0], pos.ctypes.data_as(C.c_void_p),
                           vel.ctypes.data_as(C.c_void_p), last.ctypes.data_as(C.c_void_p), C.c_double(dt),
                           C.c_double(eps), int(it))


def _rattle(c, pos, vel, dt, virial=None):
    a = np.ascontiguousarray(c["atoms"], np.int32)
    r = np.ascontiguousarray(c["rest"], np.float64)
    m = np.ascontiguousarray(c["mass"], np.float64)
    eps, it = c["rattle"]
    return lib().pmo_rattle(len(r), a.ctypes.data_as(C.c_void_p), r.ctypes.data_as(C.c_void_p),
                            m.ctypes.data_as(C.c_void_p), pos.ctypes.data_as(C.c_void_p),
                            vel.ctypes.data_as(C.c_void_p), C.c_double(dt), C.c_double(eps), int(it),
                            None if virial is None else virial.ctypes.data_as(C.c_void_p))


def leapfrog(system, specs, velocities, timestep, steps, positions=None, forces=None, constraints=None):
    """LeapfrogIntegrator::run(steps) without modifiers
    (integrators/LeapfrogIntegrator.cpp:107-120) on the oracle's forces, in the
    reference's operation order:

    * doHalfKickdoDrift (:47-68): v += F h 0.5 / m, x += v h, h = dt / T;
    * doKickdoDrift (:70-101) for the later steps: v += F h / m, x += v h;
    * calculateForces after every drift;
    * doHalfKick (StandardIntegrator.cpp:83-96) at the end: v += F h' / m,
      h' = 0.5 dt / T.

    numpy multiplies and adds without fusing them, as the reference's build
    without FMA contraction does.  ``forces`` are the forces at the starting
    positions (evaluated here when not given).  ``constraints`` ({"atoms",
    "rest", "mass", "shake": (eps, max_iter) or None, "rattle": ... or None})
    adds the SHAKE post-drift and RATTLE post-step modifiers
    (applications/protomol-app/protomol.cpp:553-577): with RATTLE the later
    steps are half kick, RATTLE, half kick, drift (:72-83), SHAKE follows
    every drift, RATTLE the final half kick; its virial then lands in the
    returned result's "virial" entry.  Returns (positions, velocities,
    forces, result of the last evaluation)."""
    x = np.array(system.positions if positions is None else positions, np.float64)
    v = np.array(velocities, np.float64)
    m = np.asarray(system.mass, np.float64)[:, None]
    r = None
    f = np.array(forces, np.float64) if forces is not None else evaluate(system, specs, positions=x)["forces"]
    h = timestep * INV_TIMEFACTOR
    hk = 0.5 * timestep * INV_TIMEFACTOR
    c = constraints
    shake = bool(c and c.get("shake"))
    rattle = bool(c and c.get("rattle"))
    dt = timestep / TIMEFACTOR
    last = x.copy() if shake else None
    for step in range(steps):
        if step > 0 and rattle:
            v = v + (f * hk) / m
            _rattle(c, x, v, dt)
            v = v + (f * hk) / m
            x = x + v * h
        else:
            if step == 0:
                v = v + ((f * h) * 0.5) / m
            else:
                v = v + (f * h) / m
            x = x + v * h
        if shake:
            _shake(c, x, v, last, dt)
        r = evaluate(system, specs, positions=x)
        f = r["forces"]
    v = v + (f * hk) / m
    if rattle:
        vir = np.zeros(9)
        _rattle(c, x, v, dt, vir)
        if r is not None:
            r["virial"] = r["virial"] + vir
    return x, v, f, r


def impulse(system, slow_specs, fast_specs, velocities, timestep, cyclelength, steps):
    """ImpulseIntegrator::run(steps) over an inner Leapfrog of ``timestep``
    without modifiers (StandardIntegrator.cpp:24-35, MTSIntegrator.cpp):
    doHalfKick with the slow forces (h = 0.5 (cyclelength dt) / T), the
    inner LeapfrogIntegrator::run(cyclelength) on the fast forces,
    calculateForces of the slow group, doHalfKick.  Returns (positions,
    velocities, slow forces, fast forces, total potential energy)."""
    x = np.array(system.positions, np.float64)
    v = np.array(velocities, np.float64)
    m = np.asarray(system.mass, np.float64)[:, None]
    rs = evaluate(system, slow_specs, positions=x)
    rf = evaluate(system, fast_specs, positions=x)
    fs, ff = rs["forces"], rf["forces"]
    h = 0.5 * (cyclelength * timestep) * INV_TIMEFACTOR
    for _ in range(steps):
        v = v + (fs * h) / m
        x, v, ff, rf = leapfrog(system, fast_specs, v, timestep, cyclelength, positions=x, forces=ff)
        rs = evaluate(system, slow_specs, positions=x)
        fs = rs["forces"]
        v = v + (fs * h) / m
    return x, v, fs, ff, rs["lennard_jones"] + rs["coulomb"] + rf["lennard_jones"] + rf["coulomb"]
