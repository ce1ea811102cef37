"""GPU parity of libpmgpu against the oracle (the CPU restatement that is
itself pinned bit-exact to the reference, see test_oracle_golden.py).

Tolerances (from the reference-parity requirements of this path):
  * cell assignment and within-cutoff pair set: bit-exact;
  * FP64 kernels: forces within 1e-9 of the force RMS, energies / virial
    within 1e-10 relative;
  * mixed precision: relative RMS force error <= 1e-5 (the headline
    criterion).  On the 14,281-atom cutoff + PME metric system the total
    energy and the virial are within 1e-7 relative of the FP64 oracle: the
    energies of the pairs closer than 5 A, which carry nearly all of the FP32
    rounding there, are evaluated in FP64 (measured: 1e-8 energy, 6e-8
    virial).  On the small systems here (300 - 1,260 atoms) the total energy
    is within 1e-7 of |E_LJ| + |E_Coulomb| (measured at most 3.5e-8) and the
    virial within 1e-6 of its largest entry (at most 4e-7), except for the
    forces that are Coulomb alone or plain Coulomb: a plain Coulomb term
    gives every pair inside the cutoff an O(1) kcal/mol energy whose FP32
    rounding (a few 2^-24 each, unbiased) is not averaged down over a few
    hundred atoms, and a Coulomb-only total is a cancellation of such terms:
    2e-6 there (measured 8.3e-7 on water216_c2, 3.7e-7 small_c2_fused,
    1.3e-7 small_c2lj_c1coul).  The FP64 kernels meet 1e-10.
"""
import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import _lib
from protomol_b200 import forces as F
from protomol_b200 import systems, workloads

pytestmark = pytest.mark.gpu

MIXED_FORCE_RTOL = 1e-5
MIXED_ENERGY_RTOL = 1e-7           # relative to |E_LJ| + |E_Coulomb|
COULOMB_ONLY_ENERGY_RTOL = 2e-6    # plain Coulomb or Coulomb alone, a few hundred atoms
MIXED_VIRIAL_RTOL = 1e-6           # relative to the largest virial entry, a few hundred atoms
MIXED_METRIC_ENERGY_RTOL = 1e-7    # the 14,281-atom cutoff + PME system, relative to |E_total|
FP64_FORCE_RTOL = 1e-9
FP64_ENERGY_RTOL = 1e-10


def gpu_eval(system, defs, precision, positions=None, virial=True):
    topo = F.Topology(system)
    fs = [F.ForceFactory.make(topo, d, precision) for d in defs]
    pos = system.positions if positions is None else positions
    out = np.zeros((system.n_atoms, 3))
    e = F.ScalarStructure(virial=virial)
    F.evaluate_group(topo, fs, pos, out, e)
    return topo, fs, out, e


def rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def small_chain():
    return systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)


PME_FULL = ("Coulomb -algorithm PMEwald -real -reciprocal -correction -interpolation BSpline "
            "-gridsize 24 24 24 -cutoff 9 -alpha 0.35")
EWALD_REAL_9 = ("CoulombEwaldReal -switchingFunction Cutoff -algorithm NonbondedCutoff -cutoff 9 -alpha 0.35 "
                "-cutoff 9")


CASES = {
    "water216_c2": (systems.water_box_216, workloads.water216().forces),
    "small_split_pme": (small_chain, [workloads.lj_ewald_split(7, 9, 0.35),
                                      workloads.pme_reciprocal((24, 24, 24), 9, 0.35)]),
    "small_c1lj_ewald": (small_chain, ["LennardJones CoulombEwaldReal -switchingFunction C1 -switchingFunction Cutoff "
                                       "-algorithm NonbondedCutoff -cutoff 9 -alpha 0.35 -cutoff 9 -cutoff 9"]),
    "small_c2lj_c1coul": (small_chain, ["LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 "
                                        "-algorithm NonbondedCutoff -switchon 7 -cutoff 10 -cutoff 8 -cutoff 10"]),
    "small_c2lj_shiftcoul": (small_chain, ["LennardJones Coulomb -switchingFunction C2 -switchingFunction Shift "
                                           "-algorithm NonbondedCutoff -switchon 7 -cutoff 9 -cutoff 10 -cutoff 10"]),
    "small_cutlj_cutewald": (small_chain, ["LennardJones CoulombEwaldReal -switchingFunction Cutoff "
                                           "-switchingFunction Cutoff -algorithm NonbondedCutoff -cutoff 8 -alpha 0.35 "
                                           "-cutoff 9 -cutoff 9"]),
    "small_c2_fused": (small_chain, ["LennardJones Coulomb -switchingFunction C2 -switchingFunction C2 -algorithm "
                                     "NonbondedCutoff -switchon 8 -cutoff 9 -switchon 6 -cutoff 9 -cutoff 9"]),
    "small_shift_lj": (small_chain, ["LennardJones -switchingFunction Shift -algorithm NonbondedCutoff -cutoff 9 "
                                     "-cutoff 9"]),
    "small_cutoff_coulomb": (small_chain, ["Coulomb -switchingFunction Cutoff -algorithm NonbondedCutoff -cutoff 9 "
                                           "-cutoff 9"]),
    "small_pme_default_alpha": (small_chain, ["Coulomb -algorithm PMEwald -reciprocal -correction -interpolation "
                                              "BSpline -gridsize 25 27 30 -cutoff 9"]),
    "smallbox_wrap": (lambda: systems.water_box(100, seed=7), workloads.water_box_workload(100, 7).forces),
    # realTerm on the GPU: the whole PME force in one keyword (box edge 24 > 2 Rc)
    "small_pme_full": (small_chain, [PME_FULL]),
}


# the cases whose forces are plain Coulomb or Coulomb alone
COULOMB_ONLY = {"water216_c2", "small_c2_fused", "small_c2lj_c1coul", "small_c2lj_shiftcoul",
                "small_cutoff_coulomb", "small_pme_full"}


def energy_scale(r):
    return abs(r["lennard_jones"]) + abs(r["coulomb"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_forces_energies_virial_against_oracle(name, precision):
    factory, defs = CASES[name]
    s = factory()
    ref = oracle.evaluate(s, [F.parse_definition(d) for d in defs])
    _, _, f, e = gpu_eval(s, defs, precision)
    scale = energy_scale(ref)
    vscale = np.abs(ref["virial"]).max()
    if precision == "fp64":
        rms = np.sqrt((ref["forces"] ** 2).sum(1).mean())
        assert np.abs(f - ref["forces"]).max() <= FP64_FORCE_RTOL * rms
        assert abs(e.lennard_jones - ref["lennard_jones"]) <= FP64_ENERGY_RTOL * scale
        assert abs(e.coulomb - ref["coulomb"]) <= FP64_ENERGY_RTOL * scale
        assert np.abs(e.virial_tensor - ref["virial"]).max() <= FP64_ENERGY_RTOL * vscale
    else:
        assert rel_rms(f, ref["forces"]) <= MIXED_FORCE_RTOL
        etot = e.lennard_jones + e.coulomb
        rtot = ref["lennard_jones"] + ref["coulomb"]
        etol = COULOMB_ONLY_ENERGY_RTOL if name in COULOMB_ONLY else MIXED_ENERGY_RTOL
        assert abs(etot - rtot) <= etol * scale
        assert np.abs(e.virial_tensor - ref["virial"]).max() <= MIXED_VIRIAL_RTOL * vscale


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_chain14281_metric_config(chain14281, precision):
    w = workloads.chain14281()
    ref = oracle.evaluate(chain14281, [F.parse_definition(d) for d in w.forces])
    _, _, f, e = gpu_eval(chain14281, w.forces, precision)
    err = rel_rms(f, ref["forces"])
    scale = energy_scale(ref)
    etot = e.lennard_jones + e.coulomb
    rtot = ref["lennard_jones"] + ref["coulomb"]
    print(f"\n{precision}: force rel RMS {err:.3e}  total energy rel {abs(etot - rtot) / abs(rtot):.3e} "
          f"(scale {abs(etot - rtot) / scale:.3e})  LJ {e.lennard_jones:.9f}/{ref['lennard_jones']:.9f} "
          f"Coul {e.coulomb:.9f}/{ref['coulomb']:.9f}")
    if precision == "fp64":
        assert err <= FP64_FORCE_RTOL
        assert abs(etot - rtot) <= FP64_ENERGY_RTOL * scale
    else:
        assert err <= MIXED_FORCE_RTOL
        assert abs(etot - rtot) <= MIXED_METRIC_ENERGY_RTOL * abs(rtot)
        dv = e.virial_tensor - ref["virial"]
        assert np.linalg.norm(dv) <= MIXED_METRIC_ENERGY_RTOL * np.linalg.norm(ref["virial"])


@pytest.mark.parametrize("name", ["water_box_216", "chain_in_water_14281"])
def test_cell_assignment_bit_exact(name):
    s = getattr(systems, name)()
    for pos in (s.positions, s.positions + np.array([40.1, -77.7, 13.3])):
        topo, _, _, _ = gpu_eval(s, [workloads.water216().forces[0]], "mixed", positions=pos)
        cells, dims = topo.cells()
        ocells, odims, _ = oracle.cell_assign(s, pos)
        assert dims == odims
        assert np.array_equal(cells, ocells)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["water216", "chain14281", "wrap", "c2_fused", "pme_real"])
def test_pair_set_bit_exact(case, precision, chain14281):
    oracle_def = None
    if case == "pme_real":
        # the real-space pairs of PMEwald -real are those of the Ewald-real
        # cutoff force at the same cutoff (realTerm with no lattice images)
        s, d, oracle_def = small_chain(), PME_FULL, EWALD_REAL_9
    elif case == "water216":
        s, d = systems.water_box_216(), workloads.water216().forces[0]
    elif case == "chain14281":
        s, d = chain14281, workloads.chain14281().forces[0]
    elif case == "wrap":
        s, d = systems.water_box(100, seed=7), workloads.water_box_workload(100, 7).forces[0]
    else:
        s, d = small_chain(), CASES["small_c2_fused"][1][0]
    topo = F.Topology(s)
    force = F.ForceFactory.make(topo, d, precision)
    gp = force.pairs(s.positions)
    op = oracle.evaluate(s, [F.parse_definition(oracle_def or d)], want_pairs=True)["pairs"]
    key = lambda p: np.sort(p[:, 0].astype(np.int64) * s.n_atoms + p[:, 1])
    assert len(gp) == len(op)
    assert np.array_equal(key(gp), key(op))


def test_pairs_near_the_cutoff_are_decided_in_fp64():
    """Atoms placed at distances rc(1 +- 1e-9): the FP32 distance cannot tell
    them apart, the FP64 re-decision must."""
    s = systems.water_box_216()
    pos = s.positions.copy()
    rc = 9.0
    rng = np.random.default_rng(5)
    for k, i in enumerate(range(0, 600, 60)):
        j = i + 30
        direction = rng.normal(size=3)
        direction /= np.linalg.norm(direction)
        pos[j] = pos[i] + direction * rc * (1 + (1e-9 if k % 2 else -1e-9))
    d = workloads.water216().forces[0]
    topo = F.Topology(s)
    force = F.ForceFactory.make(topo, d, "mixed")
    gp = force.pairs(pos)
    op = oracle.evaluate(s, [F.parse_definition(d)], positions=pos, want_pairs=True)["pairs"]
    key = lambda p: np.sort(p[:, 0].astype(np.int64) * s.n_atoms + p[:, 1])
    assert np.array_equal(key(gp), key(op))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_deterministic_and_accumulating(precision, small_chain):
    defs = CASES["small_split_pme"][1]
    topo = F.Topology(small_chain)
    fs = [F.ForceFactory.make(topo, d, precision) for d in defs]
    out1 = np.zeros((small_chain.n_atoms, 3))
    e1 = F.ScalarStructure()
    F.evaluate_group(topo, fs, small_chain.positions, out1, e1)
    out2 = np.ones((small_chain.n_atoms, 3))
    e2 = F.ScalarStructure()
    e2.lennard_jones = 5.0
    F.evaluate_group(topo, fs, small_chain.positions, out2, e2)
    # fixed-point sums are order independent: bitwise identical reruns
    assert np.array_equal(out2 - 1.0, (out1 + 1.0) - 1.0)
    assert e2.lennard_jones - 5.0 == pytest.approx(e1.lennard_jones, rel=1e-15)
    out3 = np.zeros((small_chain.n_atoms, 3))
    F.evaluate_group(topo, fs, small_chain.positions, out3, F.ScalarStructure())
    assert np.array_equal(out1, out3)


def test_virial_only_when_requested(small_chain):
    _, _, _, e = gpu_eval(small_chain, CASES["small_split_pme"][1], "mixed", virial=False)
    assert not e.virial_tensor.any()


def test_overlapping_atoms_report_overflow():
    s = systems.water_box_216()
    pos = s.positions.copy()
    pos[3] = pos[0]          # two oxygens of different waters on top of each other
    with pytest.raises(_lib.PmgpuError) as ei:
        gpu_eval(s, workloads.water216().forces, "mixed", positions=pos)
    assert ei.value.code == 3


def test_empty_and_sparse_systems():
    s = systems.water_box_216()
    empty = s.copy()
    empty.positions = np.zeros((0, 3))
    empty.scaled_charge = np.zeros(0)
    empty.atom_type = np.zeros(0, np.int32)
    empty.molecule = np.zeros(0, np.int32)
    empty.mass = np.zeros(0)
    empty.exclusions = np.zeros((0, 3), np.int32)
    empty.exclusion_check = np.zeros(0, np.int32)
    _, _, f, e = gpu_eval(empty, workloads.water216().forces, "mixed")
    assert f.shape == (0, 3) and e.lennard_jones == 0.0 and e.coulomb == 0.0
    # three waters in the big box: almost every cell empty (ragged cells)
    sparse = s.copy()
    keep = np.arange(9)
    sparse.positions = s.positions[keep] * np.array([1.0, 1.0, 1.0])
    sparse.positions[3:6] += 2.0
    sparse.scaled_charge = s.scaled_charge[keep]
    sparse.atom_type = s.atom_type[keep]
    sparse.molecule = s.molecule[keep]
    sparse.mass = s.mass[keep]
    m = (s.exclusions[:, 0] < 9) & (s.exclusions[:, 1] < 9)
    sparse.exclusions = s.exclusions[m]
    sparse.exclusion_check = s.exclusion_check[m]
    for precision in ("fp64", "mixed"):
        ref = oracle.evaluate(sparse, [F.parse_definition(d) for d in workloads.water216().forces])
        _, _, f, e = gpu_eval(sparse, workloads.water216().forces, precision)
        assert rel_rms(f, ref["forces"]) <= MIXED_FORCE_RTOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pme_real_with_lattice_images_against_oracle(precision):
    """A box under twice the cutoff: realTerm sums the lattice images of every
    pair (and of every atom with itself) besides the minimal one."""
    s = systems.water_box(100, seed=7)           # edge < 2 x 9 A
    assert min(s.box[k][k] for k in range(3)) < 18.0
    d = PME_FULL.replace("-gridsize 24 24 24", "-gridsize 16 16 16")
    ref = oracle.evaluate(s, [F.parse_definition(d)])
    _, _, f, e = gpu_eval(s, [d], precision)
    rms = np.sqrt((ref["forces"] ** 2).sum(1).mean())
    if precision == "fp64":
        assert np.abs(f - ref["forces"]).max() <= FP64_FORCE_RTOL * rms
        assert abs(e.coulomb - ref["coulomb"]) <= FP64_ENERGY_RTOL * abs(ref["coulomb"])
        assert np.abs(e.virial_tensor - ref["virial"]).max() <= FP64_ENERGY_RTOL * np.abs(ref["virial"]).max()
    else:
        # the lattice real space is FP64 in both precisions; the reciprocal
        # part is the mixed one
        assert rel_rms(f, ref["forces"]) <= MIXED_FORCE_RTOL
        assert abs(e.coulomb - ref["coulomb"]) <= MIXED_METRIC_ENERGY_RTOL * abs(ref["coulomb"])
    # the real-space term alone, where the images matter most
    dr = "Coulomb -algorithm PMEwald -real -interpolation BSpline -gridsize 16 16 16 -cutoff 9 -alpha 0.35"
    ref = oracle.evaluate(s, [F.parse_definition(dr)])
    _, _, f, e = gpu_eval(s, [dr], precision)
    assert np.abs(f - ref["forces"]).max() <= FP64_FORCE_RTOL * rms
    assert abs(e.coulomb - ref["coulomb"]) <= FP64_ENERGY_RTOL * abs(ref["coulomb"])


def test_pme_rejects_what_the_reference_rejects(small_chain):
    topo = F.Topology(small_chain)
    for bad in ("Coulomb -algorithm PMEwald -reciprocal -correction -interpolation BSpline -gridsize 24 24 24 "
                "-cutoff 9 -order 3",
                "Coulomb -algorithm PMEwald -reciprocal -correction -interpolation BSpline -gridsize 2 24 24 -cutoff 9"):
        with pytest.raises(_lib.PmgpuError) as ei:
            F.ForceFactory.make(topo, bad)
        assert ei.value.code == 1


def test_pme_default_alpha_matches_reference_bisection(small_chain):
    topo = F.Topology(small_chain)
    f = F.ForceFactory.make(topo, CASES["small_pme_default_alpha"][1][0])
    r = oracle.evaluate(small_chain, [F.parse_definition(CASES["small_pme_default_alpha"][1][0])])
    assert f.alpha == r["alpha"] == systems.ewald_alpha(9.0)


def test_million_atom_cutoff_force_fp64_against_oracle():
    """The FP64 kernels on the whole 1,000,000-atom cutoff force against the
    oracle (3.6e8 pairs, ~30 s on one host core): energies and forces."""
    w = workloads.water1m()
    s = w.system
    ref = oracle.evaluate(s, [F.parse_definition(w.forces[0])])
    _, _, f, e = gpu_eval(s, [w.forces[0]], "fp64")
    rms = np.sqrt((ref["forces"] ** 2).sum(1).mean())
    print(f"\n1M cutoff force FP64: dLJ {e.lennard_jones - ref['lennard_jones']:+.2e}  "
          f"dC {e.coulomb - ref['coulomb']:+.2e}  max |dF| / rms {np.abs(f - ref['forces']).max() / rms:.2e}")
    scale = abs(ref["lennard_jones"]) + abs(ref["coulomb"])
    assert abs(e.lennard_jones - ref["lennard_jones"]) <= FP64_ENERGY_RTOL * scale
    assert abs(e.coulomb - ref["coulomb"]) <= FP64_ENERGY_RTOL * scale
    assert np.abs(f - ref["forces"]).max() <= FP64_FORCE_RTOL * rms
    assert np.abs(e.virial_tensor - ref["virial"]).max() <= FP64_ENERGY_RTOL * np.abs(ref["virial"]).max()


def test_million_atom_box_at_full_size():
    """The 1,000,000-atom configuration (333,333 waters + Na+, 215.4 A, cutoff
    12, PME 216^3) at full size, through size-independent properties: the
    binning is bit-exact with the oracle's cell assignment, and the mixed
    path agrees with the FP64 kernels (themselves pinned to the oracle on the
    smaller systems) within the mixed tolerances."""
    w = workloads.water1m()
    s = w.system
    assert s.n_atoms == 1_000_000
    topo_m, _, fm, em = gpu_eval(s, w.forces, "mixed")
    topo_m_layout = topo_m.pair_layout()
    cells, dims = topo_m.cells()
    ocells, odims, _ = oracle.cell_assign(s, s.positions)
    assert dims == odims and np.array_equal(cells, ocells)
    topo_m.close()
    _, _, fd, ed = gpu_eval(s, w.forces, "fp64")
    assert np.isfinite(fm).all() and np.abs(fd).max() > 0
    assert rel_rms(fm, fd) <= MIXED_FORCE_RTOL
    assert np.abs(em.virial_tensor - ed.virial_tensor).max() <= MIXED_VIRIAL_RTOL * np.abs(ed.virial_tensor).max()
    etot, dtot = em.lennard_jones + em.coulomb, ed.lennard_jones + ed.coulomb
    print(f"\n1M: force rel RMS {rel_rms(fm, fd):.2e}  total energy rel {abs(etot - dtot) / abs(dtot):.2e}  "
          f"LJ rel {abs(em.lennard_jones - ed.lennard_jones) / abs(ed.lennard_jones):.2e}  virial frob rel "
          f"{np.linalg.norm(em.virial_tensor - ed.virial_tensor) / np.linalg.norm(ed.virial_tensor):.2e}")
    # 216^3 takes FP64 B-spline weights and an FP64 forward transform for the
    # reciprocal energy and virial.  The total energy (-35,145 kcal/mol, a
    # tenfold cancellation of the LJ, real-space, reciprocal and self terms)
    # holds the metric-system bound: the column layout's fixed-point pair
    # vectors carry no shared rounding into the FP32 pair energies
    assert topo_m_layout == "columns"
    assert abs(em.lennard_jones - ed.lennard_jones) <= MIXED_METRIC_ENERGY_RTOL * abs(ed.lennard_jones)
    assert abs(etot - dtot) <= MIXED_METRIC_ENERGY_RTOL * abs(dtot)
    assert np.linalg.norm(em.virial_tensor - ed.virial_tensor) <= \
        MIXED_METRIC_ENERGY_RTOL * np.linalg.norm(ed.virial_tensor)
