"""The molecular virial (ScalarStructure::molecularVirial()) on the GPU
against the oracle, which the compiled reference pins
(tests/test_oracle_vs_reference.py::test_molecular_virial_against_reference).

ProtoMol's terms: every pair of atoms of different molecules adds its force
against the minimal difference of the molecules' positions
(OneAtomPair.h:174-181, realTerm NonbondedPMEwaldSystemForce.h:750-757), the
reciprocal term adds scalarSum's tensor (Grid.h:378-386) and every atom's
reciprocal force against its offset from its molecule's position
(reciprocalTerm, :903-924).  The pair part is recomputed in FP64 in both
precisions; in mixed precision the reciprocal part carries the FP32 grid's
force error, so the bound there is 1e-6 of the tensor's largest entry
(FP64: 1e-10).
"""
import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import _lib
from protomol_b200 import forces as F
from protomol_b200 import systems, workloads

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10
MIXED_RTOL = 1e-6

PME_CHAIN = ("Coulomb -algorithm PMEwald -real -reciprocal -correction -interpolation BSpline "
             "-gridsize 24 24 24 -cutoff 9 -alpha 0.35")
LJ_C2 = "LennardJones -algorithm NonbondedCutoff -switchingFunction C2 -switchon 8 -cutoff 9"


def cases():
    water = systems.perturbed(systems.water_box_216(), 0.3, 1)
    chain = systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)
    small = systems.water_box(100, seed=7)
    return {
        "water216_cutoff": (water, workloads.water216().forces),
        "chain_pme_lj": (chain, [PME_CHAIN, LJ_C2]),
        "lattice_pme": (small, [PME_CHAIN.replace("-gridsize 24 24 24", "-gridsize 16 16 16")]),
        "chain_coulomb_c1": (chain, ["Coulomb -algorithm NonbondedCutoff -switchingFunction C1 -cutoff 9"]),
    }


def gpu_molvir(s, defs, precision, virial, com):
    topo = F.Topology(s)
    fs = [F.ForceFactory.make(topo, d, precision) for d in defs]
    topo.set_molecule_positions(com)
    out = np.zeros((s.n_atoms, 3))
    e = F.ScalarStructure(virial=virial, molecular_virial=True)
    F.evaluate_group(topo, fs, s.positions, out, e)
    return topo, out, e


def rel_max(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("virial", [True, False])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["water216_cutoff", "chain_pme_lj", "lattice_pme", "chain_coulomb_c1"])
def test_molecular_virial_against_oracle(case, precision, virial):
    s, defs = cases()[case]
    com = F.molecular_centers(s.molecule, s.positions)
    ref = oracle.evaluate(s, [F.parse_definition(d) for d in defs], mol_pos=com, virial=virial)
    _, f, e = gpu_molvir(s, defs, precision, virial, com)
    dm = rel_max(e.molecular_virial_tensor, ref["mol_virial"])
    dv = rel_max(e.virial_tensor, ref["virial"])
    print(f"\n{case} {precision} virial={virial}: molecular virial {dm:.2e}, virial {dv:.2e}")
    tol = FP64_RTOL if precision == "fp64" else MIXED_RTOL
    assert dm <= tol
    # the atomic virial keeps its own bounds (tests/test_gpu_parity.py); with
    # virial() off it is the FP64 inter-molecular pair part alone
    assert dv <= (FP64_RTOL if (precision == "fp64" or not virial) else 2e-6)
    # the forces do not change with the molecular virial
    rms = np.sqrt((ref["forces"] ** 2).sum(1).mean())
    if precision == "fp64":
        assert np.abs(f - ref["forces"]).max() <= 1e-9 * rms


def test_molecular_virial_on_the_column_layout():
    """The 9,000-atom box of the batched-water configuration, whose mixed
    cutoff force takes the column layout: the molecular virial kernels read
    the cell-sorted order binned beside it."""
    ws = workloads.batched96()
    w = ws[int(np.argmax([x.system.n_atoms for x in ws]))]
    s = w.system
    com = F.molecular_centers(s.molecule, s.positions)
    ref = oracle.evaluate(s, [F.parse_definition(d) for d in w.forces], mol_pos=com)
    topo, _, e = gpu_molvir(s, w.forces, "mixed", True, com)
    assert topo.pair_layout() == "columns"
    dm = rel_max(e.molecular_virial_tensor, ref["mol_virial"])
    print(f"\ncolumns, {s.n_atoms} atoms: molecular virial {dm:.2e}")
    assert dm <= MIXED_RTOL


def test_molecular_virial_follows_the_molecule_positions():
    """The positions are the caller's (ProtoMol's molecules[m].position): a
    shift of every molecule position by a lattice vector changes nothing,
    a shift by half an edge changes the minimal differences."""
    s, defs = cases()["chain_pme_lj"]
    com = F.molecular_centers(s.molecule, s.positions)
    L = s.box[0][0]
    _, _, e0 = gpu_molvir(s, defs, "fp64", True, com)
    _, _, e1 = gpu_molvir(s, defs, "fp64", True, com + np.array([L, -L, 2 * L]))
    assert rel_max(e1.molecular_virial_tensor, e0.molecular_virial_tensor) <= 1e-12
    moved = com.copy()
    moved[::2, 0] += 0.5 * L
    ref = oracle.evaluate(s, [F.parse_definition(d) for d in defs], mol_pos=moved)
    _, _, e2 = gpu_molvir(s, defs, "fp64", True, moved)
    assert rel_max(e2.molecular_virial_tensor, ref["mol_virial"]) <= FP64_RTOL
    assert rel_max(e2.molecular_virial_tensor, e0.molecular_virial_tensor) > 1e-3


def test_molecular_virial_errors():
    s, defs = cases()["chain_pme_lj"]
    topo = F.Topology(s)
    fs = [F.ForceFactory.make(topo, d, "mixed") for d in defs]
    out = np.zeros((s.n_atoms, 3))
    with pytest.raises(_lib.PmgpuError) as ex:
        F.evaluate_group(topo, fs, s.positions, out, F.ScalarStructure(molecular_virial=True))
    assert ex.value.code == 4                       # no molecule positions yet
    with pytest.raises(_lib.PmgpuError) as ex:
        topo.set_molecule_positions(np.zeros((3, 3)))
    assert ex.value.code == 1                       # one per molecule
    v = systems.vacuum_chain_104()
    tv = F.Topology(v)
    full = F.ForceFactory.make(tv, "LennardJones Coulomb -algorithm NonbondedSimpleFull", "fp64")
    tv.set_molecule_positions(F.molecular_centers(v.molecule, v.positions))
    with pytest.raises(_lib.PmgpuError) as ex:
        F.evaluate_group(tv, [full], v.positions, np.zeros((v.n_atoms, 3)), F.ScalarStructure(molecular_virial=True))
    assert ex.value.code == 5
