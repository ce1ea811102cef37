"""The column-cluster layout of the mixed pair forces (boxes well above twice
the cutoff) against the oracle, pairing by pairing.

Every registered OneAtomPair[Two] pairing of the parity suite runs here on a
40 A box of 6,400 atoms (a 100-atom chain in 2,100 waters), where the mixed
cutoff forces take the column layout: fixed-point coordinates whose int32
differences are the exact minimal-image displacements, z-sorted columns,
8 x 4 tiles.  Bounds: the within-cutoff pair set bit-exact; forces within
1e-5 relative RMS; total energy and virial within 1e-7 of the FP64 oracle
(|E_LJ| + |E_Coulomb| and the virial's largest entry as the scales), except:

* a plain Coulomb term gives every pair inside the cutoff an O(1) kcal/mol
  energy, so its FP32 rounding (a few 2^-24 per pair) is spread over all
  pairs: 4e-7 on the energy there (1.4e-7 measured, lj_c2_coul_c2);
* the virial of a Coulomb-only force (plain, tabulated or Ewald real space
  alone) is a near cancellation of its pair terms, the largest of them the
  FP32 forces of the hydrogen-bonded pairs: 2e-6 there (1.35e-6 measured,
  Ewald real space alone; 5e-8 with the Lennard-Jones term beside it).
"""
import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import forces as F
from protomol_b200 import systems, workloads

pytestmark = pytest.mark.gpu

FORCE_RTOL = 1e-5
ENERGY_RTOL = 1e-7
PLAIN_COULOMB_ENERGY_RTOL = 4e-7
COULOMB_ONLY_VIRIAL_RTOL = 2e-6


def medium_chain():
    return systems.chain_in_water(n_chain=100, n_water=2100, length=40.0, seed=12)


PAIRINGS = {
    "lj_c2_ewald": workloads.lj_ewald_split(7, 9, 0.35),
    "lj_c1_ewald": "LennardJones CoulombEwaldReal -switchingFunction C1 -switchingFunction Cutoff "
                   "-algorithm NonbondedCutoff -cutoff 9 -alpha 0.35 -cutoff 9 -cutoff 9",
    "lj_cut_ewald_cut": "LennardJones CoulombEwaldReal -switchingFunction Cutoff -switchingFunction Cutoff "
                        "-algorithm NonbondedCutoff -cutoff 8 -alpha 0.35 -cutoff 9 -cutoff 9",
    "lj_c2_coul_c1": "LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 "
                     "-algorithm NonbondedCutoff -switchon 7 -cutoff 10 -cutoff 8 -cutoff 10",
    "lj_c2_coul_shift": "LennardJones Coulomb -switchingFunction C2 -switchingFunction Shift "
                        "-algorithm NonbondedCutoff -switchon 7 -cutoff 9 -cutoff 10 -cutoff 10",
    "lj_c2_coul_c2": "LennardJones Coulomb -switchingFunction C2 -switchingFunction C2 -algorithm "
                     "NonbondedCutoff -switchon 8 -cutoff 9 -switchon 6 -cutoff 9 -cutoff 9",
    "lj_shift": "LennardJones -switchingFunction Shift -algorithm NonbondedCutoff -cutoff 9 -cutoff 9",
    "coul_cutoff": "Coulomb -switchingFunction Cutoff -algorithm NonbondedCutoff -cutoff 9 -cutoff 9",
    "ewald_cutoff": "CoulombEwaldReal -switchingFunction Cutoff -algorithm NonbondedCutoff -cutoff 9 -alpha 0.35 "
                    "-cutoff 9",
    "ljtable_ewaldtable": "LennardJonesTable CoulombEwaldRealTable -switchingFunction C2 -algorithm NonbondedCutoff "
                          "-switchon 7 -cutoff 9 -cutoff 9 -alpha 0.35 -cutoff 9",
    "coultable_shift": "CoulombTable -switchingFunction Shift -algorithm NonbondedCutoff -cutoff 9 -cutoff 9",
}
PLAIN_COULOMB = {"lj_c2_coul_c1", "lj_c2_coul_shift", "lj_c2_coul_c2", "coul_cutoff", "coultable_shift"}
COULOMB_ONLY = {"coul_cutoff", "ewald_cutoff", "coultable_shift"}


@pytest.fixture(scope="module")
def medium():
    return medium_chain()


def _eval(s, defs, precision, positions=None):
    topo = F.Topology(s)
    fs = [F.ForceFactory.make(topo, d, precision) for d in defs]
    out = np.zeros((s.n_atoms, 3))
    e = F.ScalarStructure(virial=True)
    F.evaluate_group(topo, fs, s.positions if positions is None else positions, out, e)
    return topo, fs, out, e


def _rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


@pytest.mark.parametrize("name", sorted(PAIRINGS))
def test_column_layout_against_oracle(medium, name):
    d = PAIRINGS[name]
    ref = oracle.evaluate(medium, [F.parse_definition(d)])
    topo, fs, f, e = _eval(medium, [d], "mixed")
    assert topo.pair_layout() == "columns"
    scale = abs(ref["lennard_jones"]) + abs(ref["coulomb"])
    de = abs((e.lennard_jones + e.coulomb) - (ref["lennard_jones"] + ref["coulomb"])) / scale
    dv = np.abs(e.virial_tensor - ref["virial"]).max() / np.abs(ref["virial"]).max()
    err = _rel_rms(f, ref["forces"])
    print(f"\n{name}: force {err:.2e} energy {de:.2e} virial {dv:.2e}")
    tol = PLAIN_COULOMB_ENERGY_RTOL if name in PLAIN_COULOMB else ENERGY_RTOL
    assert err <= FORCE_RTOL
    assert de <= tol
    assert dv <= (COULOMB_ONLY_VIRIAL_RTOL if name in COULOMB_ONLY else tol)
    # the pair set of the column layout is the reference's, bit for bit
    gp = fs[0].pairs(medium.positions)
    op = oracle.evaluate(medium, [F.parse_definition(d)], want_pairs=True)["pairs"]
    key = lambda p: np.sort(p[:, 0].astype(np.int64) * medium.n_atoms + p[:, 1])
    assert len(gp) == len(op) and np.array_equal(key(gp), key(op))


def test_column_layout_split_pme_and_reruns_are_bitwise(medium):
    defs = [workloads.lj_ewald_split(7, 9, 0.35), workloads.pme_reciprocal((40, 40, 40), 9, 0.35)]
    ref = oracle.evaluate(medium, [F.parse_definition(d) for d in defs])
    topo, fs, f, e = _eval(medium, defs, "mixed")
    assert topo.pair_layout() == "columns"
    etot, rtot = e.lennard_jones + e.coulomb, ref["lennard_jones"] + ref["coulomb"]
    assert _rel_rms(f, ref["forces"]) <= FORCE_RTOL
    assert abs(etot - rtot) <= ENERGY_RTOL * abs(rtot)
    assert np.linalg.norm(e.virial_tensor - ref["virial"]) <= ENERGY_RTOL * np.linalg.norm(ref["virial"])
    f2 = np.zeros_like(f)
    e2 = F.ScalarStructure()
    F.evaluate_group(topo, fs, medium.positions, f2, e2)
    assert np.array_equal(f, f2) and e.lennard_jones == e2.lennard_jones and e.coulomb == e2.coulomb


def test_column_layout_pairs_near_the_cutoff_are_decided_in_fp64(medium):
    """Pairs placed at rc (1 +- 1e-9) across the box and across its periodic
    faces: the FP32 distance cannot tell them apart, the FP64 re-decision
    must, and the fixed-point minimal image must find the wrapped ones."""
    pos = medium.positions.copy()
    rc = 9.0
    L = medium.box_lengths
    rng = np.random.default_rng(9)
    chain = 100
    for k, i in enumerate(range(chain, chain + 3000, 150)):
        j = i + 75
        direction = rng.normal(size=3)
        direction /= np.linalg.norm(direction)
        pj = pos[i] + direction * rc * (1 + (1e-9 if k % 2 else -1e-9))
        if k % 3 == 0:
            pj = pj + L * rng.integers(-1, 2, size=3)       # the same point in another image
        pos[j] = pj
    d = PAIRINGS["lj_c2_ewald"]
    topo = F.Topology(medium)
    force = F.ForceFactory.make(topo, d, "mixed")
    gp = force.pairs(pos)
    assert topo.pair_layout() == "columns"
    op = oracle.evaluate(medium, [F.parse_definition(d)], positions=pos, want_pairs=True)["pairs"]
    key = lambda p: np.sort(p[:, 0].astype(np.int64) * medium.n_atoms + p[:, 1])
    assert np.array_equal(key(gp), key(op))


def test_dilute_columns_fall_back_to_the_cell_layout():
    """A dilute gas in a box only a little over twice the cutoff high: an
    8-atom cluster of a column spans more of the height than the column
    layout allows (a tile's periodic image could be ambiguous), so the
    evaluation is redone on the cell layout, with the same results bar the
    FP32 rounding."""
    rng = np.random.default_rng(3)
    base = systems.oxygen_fluid_216()
    s = base.copy()
    n = 160
    L = np.array([44.0, 44.0, 30.0])
    # 160 of the 12 x 12 x 8 sites of a 3.67 x 3.67 x 3.75 A lattice, jittered
    sites = np.stack(np.meshgrid(np.arange(12), np.arange(12), np.arange(8), indexing="ij"), -1).reshape(-1, 3)
    pick = rng.choice(len(sites), n, replace=False)
    s.positions = (sites[pick] + 0.5) * (L / np.array([12, 12, 8])) + rng.uniform(-0.3, 0.3, size=(n, 3))
    s.scaled_charge = np.zeros(n)
    s.atom_type = np.zeros(n, np.int32)
    s.molecule = np.arange(n, dtype=np.int32)
    s.mass = np.full(n, 15.9994)
    s.exclusions = np.zeros((0, 3), np.int32)
    s.exclusion_check = np.zeros(0, np.int32)
    s.box = np.array([[L[0], 0, 0], [0, L[1], 0], [0, 0, L[2]], L / 2])
    d = "LennardJones -switchingFunction C2 -algorithm NonbondedCutoff -switchon 8 -cutoff 9 -cutoff 9"
    ref = oracle.evaluate(s, [F.parse_definition(d)])
    topo, _, f, e = _eval(s, [d], "mixed")
    assert topo.pair_layout() == "cells"
    assert _rel_rms(f, ref["forces"]) <= FORCE_RTOL
    assert abs(e.lennard_jones - ref["lennard_jones"]) <= 1e-6 * abs(ref["lennard_jones"])


def test_reference_cells_reported_by_the_column_binning(chain14281):
    topo, _, _, _ = _eval(chain14281, [workloads.chain14281().forces[0]], "mixed")
    assert topo.pair_layout() == "columns"
    cells, dims = topo.cells()
    ocells, odims, _ = oracle.cell_assign(chain14281, chain14281.positions)
    assert dims == odims and np.array_equal(cells, ocells)


def _moving(s, steps, seed=21, speed=0.01):
    """Positions of a synthetic trajectory: every atom moving along its own
    direction at ``speed`` A per step (a thermal-like drift, no dynamics)."""
    rng = np.random.default_rng(seed)
    u = rng.normal(size=s.positions.shape)
    u *= speed / np.linalg.norm(u, axis=1, keepdims=True) * rng.uniform(0.2, 1.0, size=(s.n_atoms, 1))
    return [s.positions + k * u for k in range(steps)]


def test_reused_pair_list_follows_a_moving_system(medium):
    """A pair list with a 1 A skin rebuilt every 10 evaluations, over 25
    evaluations of moving atoms: every evaluation equals a fresh one (list
    rebuilt) up to the FP32 summation order, three lists are built, and the
    last one agrees with the oracle."""
    d = PAIRINGS["lj_c2_ewald"]
    traj = _moving(medium, 25)
    topo = F.Topology(medium)
    fs = [F.ForceFactory.make(topo, d, "mixed")]
    topo.set_pair_list(1.0, 10)
    fresh = F.Topology(medium)
    ff = [F.ForceFactory.make(fresh, d, "mixed")]
    for k, pos in enumerate(traj):
        out = np.zeros((medium.n_atoms, 3)); e = F.ScalarStructure()
        F.evaluate_group(topo, fs, pos, out, e)
        ref = np.zeros((medium.n_atoms, 3)); er = F.ScalarStructure()
        F.evaluate_group(fresh, ff, pos, ref, er)
        assert _rel_rms(out, ref) <= 1e-6, k
        assert abs((e.lennard_jones + e.coulomb) - (er.lennard_jones + er.coulomb)) <= 1e-9 * (
            abs(er.lennard_jones) + abs(er.coulomb)), k
    assert topo.pair_layout() == "columns"
    assert topo.pair_list_builds() == 3
    o = oracle.evaluate(medium, [F.parse_definition(d)], positions=traj[-1])
    assert _rel_rms(out, o["forces"]) <= FORCE_RTOL
    scale = abs(o["lennard_jones"]) + abs(o["coulomb"])
    assert abs((e.lennard_jones + e.coulomb) - (o["lennard_jones"] + o["coulomb"])) <= ENERGY_RTOL * scale


def test_a_list_older_than_its_skin_is_rebuilt(medium):
    """One atom jumps 0.8 A (more than half the 1 A skin) between two
    evaluations of a reused list: the evaluation notices, rebuilds and
    repeats itself, and its result is the fresh one."""
    d = PAIRINGS["lj_c2_ewald"]
    topo = F.Topology(medium)
    fs = [F.ForceFactory.make(topo, d, "mixed")]
    topo.set_pair_list(1.0, 10)
    out = np.zeros((medium.n_atoms, 3))
    F.evaluate_group(topo, fs, medium.positions, out, F.ScalarStructure())
    pos = medium.positions.copy()
    pos[500] += np.array([0.8, 0.0, 0.0])
    out = np.zeros((medium.n_atoms, 3)); e = F.ScalarStructure()
    F.evaluate_group(topo, fs, pos, out, e)
    assert topo.pair_list_builds() == 2
    o = oracle.evaluate(medium, [F.parse_definition(d)], positions=pos)
    assert _rel_rms(out, o["forces"]) <= FORCE_RTOL
