"""Look-up-table potentials: LennardJonesTable, CoulombTable and
CoulombEwaldRealTable over LookUpTableBase (base/LookUpTableBase.h), in every
periodic combination the reference registers
(factories/registerForceExemplarsCutoff.cpp:47-48,58,69,86,101,132-134).

CPU: the definition ids and parameters; the library's table (host builder
behind pmgpu_lookup_table) equal to the oracle's bit for bit -- the oracle's
table forces are pinned bit-exact to the reference by the golden fixtures
small_*table*; the tables approximate the analytic potentials.
GPU: FP64 and mixed kernels against the oracle on a chain in water (57 1-4
pairs, coulombScalingFactor 0.5), a perturbed water box and a box small
enough for the per-pair minimal image; the 14,281-atom system with the
tabulated Ewald real part next to PME; the adjoint, HVP and dense Hessian
of the table forces."""
import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import _lib
from protomol_b200 import forces as F
from protomol_b200 import systems, workloads

MIXED_FORCE_RTOL = 1e-5
# mixed, on the small systems here: the total energy within 1e-7 of
# |E_LJ| + |E_Coulomb| and the virial within 1e-6 of its largest entry;
# forces that are plain Coulomb or Coulomb alone 2e-6 on the energy (their
# per-pair FP32 rounding is not averaged down over a few hundred atoms, and
# a Coulomb-only total is a cancellation)
MIXED_ENERGY_RTOL = 1e-7           # relative to |E_LJ| + |E_Coulomb|
COULOMB_ONLY_ENERGY_RTOL = 2e-6
MIXED_VIRIAL_RTOL = 1e-6           # relative to the largest virial entry
COULOMB_ONLY = {"coulomb_shift", "coulomb_cutoff", "ewald", "ljt_coult"}
MIXED_METRIC_ENERGY_RTOL = 1e-7    # the 14,281-atom system, relative to |E_total|
FP64_FORCE_RTOL = 1e-9
FP64_ENERGY_RTOL = 1e-10

DEFS = {
    "lj_c2": "LennardJonesTable -switchingFunction C2 -algorithm NonbondedCutoff -switchon 7 -cutoff 9 -cutoff 9",
    "coulomb_shift": "CoulombTable -switchingFunction Shift -algorithm NonbondedCutoff -cutoff 9 -cutoff 9",
    "coulomb_cutoff": "CoulombTable -switchingFunction Cutoff -algorithm NonbondedCutoff -cutoff 9 -cutoff 9",
    "ewald": "CoulombEwaldRealTable -algorithm NonbondedCutoff -cutoff 9 -alpha 0.35 -cutoff 9",
    "c2lj_ewald": ("LennardJones CoulombEwaldRealTable -switchingFunction C2 -algorithm NonbondedCutoff "
                   "-switchon 7 -cutoff 10 -cutoff 8.5 -alpha 0.35 -cutoff 10"),
    "c1lj_ewald": ("LennardJones CoulombEwaldRealTable -switchingFunction C1 -algorithm NonbondedCutoff "
                   "-cutoff 9 -cutoff 9 -alpha 0.35 -cutoff 9"),
    "cutlj_ewald": ("LennardJones CoulombEwaldRealTable -switchingFunction Cutoff -algorithm NonbondedCutoff "
                    "-cutoff 8 -cutoff 9 -alpha 0.35 -cutoff 9"),
    "ljt_ewald": ("LennardJonesTable CoulombEwaldRealTable -switchingFunction C2 -algorithm NonbondedCutoff "
                  "-switchon 8 -cutoff 9 -cutoff 10 -alpha 0.3 -cutoff 10"),
    "ljt_coult": ("LennardJonesTable CoulombTable -switchingFunction C2 -switchingFunction Shift "
                  "-algorithm NonbondedCutoff -switchon 1 -cutoff 9 -cutoff 9.5 -cutoff 9.5"),
}


# ------------------------------------------------------------------ CPU
def test_ids_and_parameters():
    t = F.parse_definition(DEFS["ljt_coult"])["terms"]
    assert t == [("C2", "LennardJonesTable", 1.0, 9.0, 0.0), ("Shift", "CoulombTable", 0.0, 9.5, 0.0)]
    assert F.cutoff_ident(t) == ("LennardJonesTable CoulombTable -switchingFunction C2 -switchingFunction Shift "
                                 "-algorithm NonbondedCutoff")
    t = F.parse_definition(DEFS["c2lj_ewald"])["terms"]
    # CoulombEwaldRealTable's tabulated Cutoff is not written in the id
    assert t == [("C2", "LennardJones", 7.0, 10.0, 0.0), ("Cutoff", "CoulombEwaldRealTable", 0.0, 8.5, 0.35)]
    assert F.cutoff_ident(t) == "LennardJones CoulombEwaldRealTable -switchingFunction C2 -algorithm NonbondedCutoff"
    assert F.parse_definition(DEFS["ewald"])["terms"] == [("Cutoff", "CoulombEwaldRealTable", 0.0, 9.0, 0.35)]
    with pytest.raises(ValueError):       # one switching function too many
        F.parse_definition("CoulombEwaldRealTable -switchingFunction Cutoff -algorithm NonbondedCutoff "
                           "-cutoff 9 -alpha 0.35 -cutoff 9")


TABLES = [("LennardJonesTable", "C2", 8.0, 9.0, 0.0), ("LennardJonesTable", "C2", 10.0, 12.0, 0.0),
          ("CoulombTable", "Shift", 0.0, 9.0, 0.0), ("CoulombTable", "Cutoff", 0.0, 12.0, 0.0),
          ("CoulombEwaldRealTable", "Cutoff", 0.0, 10.0, 0.312341327434087)]


@pytest.mark.parametrize("pot,sw,on,rc,alpha", TABLES)
def test_library_table_is_the_oracle_table(pot, sw, on, rc, alpha):
    lib = _lib.load()
    n = lib.pmgpu_lookup_table(_lib.POT[pot], _lib.SW[sw], on, rc, alpha, None, 0)
    t = np.zeros(n)
    assert lib.pmgpu_lookup_table(_lib.POT[pot], _lib.SW[sw], on, rc, alpha, t.ctypes.data, n) == n
    assert np.array_equal(t, oracle.lookup_table(pot, sw, on, rc, alpha))
    pre = 7 if pot == "LennardJonesTable" else 6
    step = 8 if pot == "LennardJonesTable" else 4
    octaves = int(np.floor(np.log2(rc * rc))) + 1 + 4          # from 2^-4 A^2
    assert n == (octaves * 2 ** pre + 1) * step


def test_unregistered_tables_are_refused():
    lib = _lib.load()
    assert lib.pmgpu_lookup_table(_lib.POT["LennardJonesTable"], _lib.SW["Shift"], 0, 9, 0, None, 0) == -1
    assert lib.pmgpu_lookup_table(_lib.POT["CoulombEwaldRealTable"], _lib.SW["C2"], 8, 9, 0.3, None, 0) == -1
    assert lib.pmgpu_lookup_table(_lib.POT["LennardJones"], _lib.SW["C2"], 8, 9, 0, None, 0) == -1


@pytest.mark.parametrize("table,analytic,etol", [
    (DEFS["lj_c2"], "LennardJones -switchingFunction C2 -algorithm NonbondedCutoff -switchon 7 -cutoff 9 -cutoff 9",
     1e-6),
    (DEFS["coulomb_shift"], "Coulomb -switchingFunction Shift -algorithm NonbondedCutoff -cutoff 9 -cutoff 9", 1e-6),
    # the table holds libm erfc, CoulombEwaldReal the poly5 approximation
    # (1.5e-7 absolute in erfc), whose per-pair differences add up against a
    # small real-space total (6.5 kcal/mol here)
    (DEFS["ewald"], "CoulombEwaldReal -switchingFunction Cutoff -algorithm NonbondedCutoff -cutoff 9 -alpha 0.35 "
                    "-cutoff 9", 1e-4),
])
def test_tables_approximate_the_analytic_potentials(table, analytic, etol):
    """The cubic Hermite interpolant in r^2 reproduces the potential it
    tabulates (except in the one interval that holds a hard cutoff)."""
    s = systems.perturbed(systems.water_box_216(), 0.3, 1)
    a = oracle.evaluate(s, [F.parse_definition(table)])
    b = oracle.evaluate(s, [F.parse_definition(analytic)])
    rms = np.sqrt((b["forces"] ** 2).sum(1).mean())
    assert np.sqrt(((a["forces"] - b["forces"]) ** 2).sum(1).mean()) <= 2e-6 * rms
    ea, eb = a["lennard_jones"] + a["coulomb"], b["lennard_jones"] + b["coulomb"]
    assert abs(ea - eb) <= etol * abs(eb)
    assert a["n_pairs"] == b["n_pairs"]


# ------------------------------------------------------------------ GPU
def _small_chain():
    return systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)


SYSTEMS = {
    "chain": _small_chain,
    "water": lambda: systems.perturbed(systems.water_box_216(), 0.3, 2),
    "smallbox": lambda: systems.water_box(100, seed=7),
}


def _gpu(system, defs, precision):
    topo = F.Topology(system)
    fs = [F.ForceFactory.make(topo, d, precision) for d in defs]
    out = np.zeros((system.n_atoms, 3))
    e = F.ScalarStructure()
    F.evaluate_group(topo, fs, system.positions, out, e)
    return out, e


def _check(system, defs, precision, etol=MIXED_ENERGY_RTOL):
    ref = oracle.evaluate(system, [F.parse_definition(d) for d in defs])
    f, e = _gpu(system, defs, precision)
    rms = np.sqrt((ref["forces"] ** 2).sum(1).mean())
    scale = abs(ref["lennard_jones"]) + abs(ref["coulomb"])
    vscale = max(np.abs(ref["virial"]).max(), 1.0)
    if precision == "fp64":
        assert np.abs(f - ref["forces"]).max() <= FP64_FORCE_RTOL * rms
        assert abs(e.lennard_jones - ref["lennard_jones"]) <= FP64_ENERGY_RTOL * scale
        assert abs(e.coulomb - ref["coulomb"]) <= FP64_ENERGY_RTOL * scale
        assert np.abs(e.virial_tensor - ref["virial"]).max() <= FP64_ENERGY_RTOL * vscale
    else:
        err = np.sqrt(((f - ref["forces"]) ** 2).sum() / (ref["forces"] ** 2).sum())
        assert err <= MIXED_FORCE_RTOL, err
        assert abs(e.lennard_jones + e.coulomb - ref["lennard_jones"] - ref["coulomb"]) <= etol * scale
        assert np.abs(e.virial_tensor - ref["virial"]).max() <= MIXED_VIRIAL_RTOL * vscale
    return ref, f, e


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", sorted(DEFS))
def test_table_forces_against_oracle(case, precision):
    _check(_small_chain(), [DEFS[case]], precision,
           COULOMB_ONLY_ENERGY_RTOL if case in COULOMB_ONLY else MIXED_ENERGY_RTOL)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("sysname", ["water", "smallbox"])
def test_table_forces_other_boxes(sysname, precision):
    s = SYSTEMS[sysname]()
    rc = 7.0 if sysname == "smallbox" else 9.0
    defs = [f"LennardJonesTable CoulombEwaldRealTable -switchingFunction C2 -algorithm NonbondedCutoff "
            f"-switchon {rc - 1} -cutoff {rc} -cutoff {rc} -alpha 0.35 -cutoff {rc}"]
    _check(s, defs, precision)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ljt_ewald", "ljt_coult", "c2lj_ewald"])
def test_table_adjoint_and_hessian(case):
    """The backward pass of a table force differentiates the cubic
    interpolant: energies equal the forward's; the charge and LJ-table
    gradients reproduce the energy through its bilinearity in the charges
    and linearity in A, B; H v against central differences of the oracle's
    forces (h = 1e-7 A, so that hardly a pair crosses an interval boundary,
    where the interpolant's second derivative jumps); the dense Hessian
    applied to v is the HVP."""
    s = _small_chain()
    d = DEFS[case]
    specs = [F.parse_definition(d)]
    topo = F.Topology(s)
    f = F.ForceFactory.make(topo, d, "fp64")
    v = np.random.default_rng(5).standard_normal((s.n_atoms, 3))
    g = F.adjoint(topo, [f], s.positions, v)
    ref = oracle.evaluate(s, specs)
    scale = abs(ref["lennard_jones"]) + abs(ref["coulomb"])
    assert abs(g["lennard_jones"] - ref["lennard_jones"]) <= 1e-10 * scale
    assert abs(g["coulomb"] - ref["coulomb"]) <= 1e-10 * scale
    assert abs(np.dot(s.scaled_charge, g["dE_dq"]) - 2.0 * ref["coulomb"]) <= 1e-9 * scale
    assert abs((s.lj_table * g["dE_dlj"]).sum() - ref["lennard_jones"]) <= 1e-9 * scale
    h = 1e-7
    fp = oracle.evaluate(s, specs, positions=s.positions + h * v)["forces"]
    fm = oracle.evaluate(s, specs, positions=s.positions - h * v)["forces"]
    hv_fd = -(fp - fm) / (2.0 * h)
    err = np.sqrt(((g["hv"] - hv_fd) ** 2).sum() / (hv_fd ** 2).sum())
    print(f"\n{case}: H v vs central differences {err:.2e}")
    assert err <= 1e-5
    H = F.hessian(topo, [f], s.positions)
    assert np.abs(H - H.T).max() <= 1e-9 * np.abs(H).max()
    hv = H @ v.ravel()
    assert np.abs(hv - g["hv"].ravel()).max() <= 1e-9 * np.abs(hv).max()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_chain14281_with_tabulated_ewald_real(precision):
    """The metric system with LennardJones C2 + CoulombEwaldRealTable (the
    reference's bpti.pme.opt configuration form) next to PME."""
    w = workloads.chain14281()
    defs = ["LennardJones CoulombEwaldRealTable -switchingFunction C2 -algorithm NonbondedCutoff "
            "-switchon 10 -cutoff 12 -cutoff 12 -alpha 0.32 -cutoff 12", w.forces[1]]
    ref = oracle.evaluate(w.system, [F.parse_definition(d) for d in defs])
    f, e = _gpu(w.system, defs, precision)
    err = np.sqrt(((f - ref["forces"]) ** 2).sum() / (ref["forces"] ** 2).sum())
    etot, rtot = e.lennard_jones + e.coulomb, ref["lennard_jones"] + ref["coulomb"]
    print(f"\n{precision}: force rel RMS {err:.2e}  dE/E {(etot - rtot) / abs(rtot):.2e}")
    if precision == "fp64":
        assert err <= FP64_FORCE_RTOL
        assert abs(etot - rtot) <= FP64_ENERGY_RTOL * (abs(ref["lennard_jones"]) + abs(ref["coulomb"]))
    else:
        assert err <= MIXED_FORCE_RTOL
        assert abs(etot - rtot) <= MIXED_METRIC_ENERGY_RTOL * abs(rtot)
