"""Live cross-check of the restatement against the compiled reference
(oracle/_ref, built from the ProtoMol sources).  Skipped where the reference
build is absent (it is never shipped with the product)."""
import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import forces as F
from protomol_b200 import systems, workloads

pytestmark = pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built here")


@pytest.mark.parametrize("seed", [1, 2])
def test_perturbed_water_bit_exact(seed):
    s = systems.perturbed(systems.water_box_216(), 0.3, seed)
    specs = [F.parse_definition(d) for d in workloads.water216().forces]
    a = oracle.evaluate(s, specs)
    b = oracle.run_reference(s, specs)
    assert np.array_equal(a["forces"], b["forces"])
    assert a["lennard_jones"] == b["lennard_jones"] and a["coulomb"] == b["coulomb"]
    assert np.array_equal(a["virial"], b["virial"])
    cells, dims, _ = oracle.cell_assign(s)
    assert np.array_equal(cells, b["cells"]) and dims == b["dims"]


def test_atoms_outside_the_box_bin_like_reference():
    s = systems.water_box_216()
    s.positions = s.positions + np.array([20.0, -37.0, 55.5])   # far outside the primary cell
    specs = [F.parse_definition(workloads.water216().forces[0])]
    a = oracle.evaluate(s, specs)
    b = oracle.run_reference(s, specs)
    assert np.array_equal(a["forces"], b["forces"])
    cells, _, _ = oracle.cell_assign(s)
    assert np.array_equal(cells, b["cells"])


def test_chain14281_split_pme_against_reference():
    w = workloads.chain14281()
    specs = [F.parse_definition(d) for d in w.forces]
    a = oracle.evaluate(w.system, specs)
    b = oracle.run_reference(w.system, specs)
    rms = np.sqrt((b["forces"] ** 2).sum(1).mean())
    assert np.abs(a["forces"] - b["forces"]).max() <= 1e-12 * rms
    assert abs(a["lennard_jones"] - b["lennard_jones"]) <= 1e-12 * abs(b["lennard_jones"])
    assert abs(a["coulomb"] - b["coulomb"]) <= 1e-9 * abs(b["coulomb"])


def charged_chain():
    """The 1,260-atom chain in water with half an elementary charge added to
    one chain atom: a non-neutral box, where PME adds the charged-system term
    -pi (sum q~)^2 / (2 V alpha^2) to the energy and the virial diagonal
    (forces/NonbondedPMEwaldSystemForce.h:604-628)."""
    s = systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)
    s.scaled_charge = s.scaled_charge.copy()
    s.scaled_charge[5] += 0.5 * systems.SQRT_COULOMB_CONSTANT
    return s


def test_charged_system_pme_against_reference():
    s = charged_chain()
    assert abs(s.scaled_charge.sum() * 0.00268283) > 1e-5      # the term is on
    d = ("Coulomb -algorithm PMEwald -real -reciprocal -correction -interpolation BSpline "
         "-gridsize 24 24 24 -cutoff 9 -alpha 0.35")
    specs = [F.parse_definition(d)]
    a = oracle.evaluate(s, specs)
    b = oracle.run_reference(s, specs)
    rms = np.sqrt((b["forces"] ** 2).sum(1).mean())
    assert np.abs(a["forces"] - b["forces"]).max() <= 1e-11 * rms
    assert abs(a["coulomb"] - b["coulomb"]) <= 1e-10 * abs(b["coulomb"])
    assert np.abs(a["virial"] - b["virial"]).max() <= 1e-10 * np.abs(b["virial"]).max()
    # the same box made neutral again differs by the charged term alone on the diagonal
    n = systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)
    c = oracle.evaluate(n, specs)
    assert c["coulomb"] != a["coulomb"]


# ---- molecular virial (ScalarStructure::molecularVirial) ----------------------
PME_CHAIN = ("Coulomb -algorithm PMEwald -real -reciprocal -correction -interpolation BSpline "
             "-gridsize 24 24 24 -cutoff 9 -alpha 0.35")
LJ_C2 = "LennardJones -algorithm NonbondedCutoff -switchingFunction C2 -switchon 8 -cutoff 9"


def molvir_cases():
    water = systems.perturbed(systems.water_box_216(), 0.3, 1)
    chain = systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)
    small = systems.water_box(100, seed=7)          # edge < 2 x 9 A: realTerm's lattice images
    return {
        "water216_cutoff": (water, workloads.water216().forces),
        "chain_pme_lj": (chain, [PME_CHAIN, LJ_C2]),
        "lattice_pme": (small, [PME_CHAIN.replace("-gridsize 24 24 24", "-gridsize 16 16 16")]),
        "chain_coulomb_c1": (chain, ["Coulomb -algorithm NonbondedCutoff -switchingFunction C1 -cutoff 9"]),
    }


@pytest.mark.parametrize("virial", [True, False])
@pytest.mark.parametrize("case", ["water216_cutoff", "chain_pme_lj", "lattice_pme", "chain_coulomb_c1"])
def test_molecular_virial_against_reference(case, virial):
    """The reference with molecularVirial() on and its molecule positions
    from buildMolecularCenterOfMass: the oracle's centres bit for bit, its
    molecular and atomic virial to the FFT's rounding.  With virial() off the
    atomic slots hold only the pairs of different molecules and the
    reciprocal tensor is missing from the molecular virial (Grid.h:341-387)."""
    s, defs = molvir_cases()[case]
    specs = [F.parse_definition(d) for d in defs]
    b = oracle.run_reference(s, specs, molecular_virial=True, virial=virial)
    com = oracle.molecular_centers(s)
    assert np.array_equal(com, b["mol_pos"])
    assert np.array_equal(F.molecular_centers(s.molecule, s.positions), com)
    a = oracle.evaluate(s, specs, mol_pos=com, virial=virial)
    pme = any(sp["kind"] == "pme" for sp in specs)
    tol = 1e-12 if pme else 0.0
    assert np.abs(a["mol_virial"] - b["mol_virial"]).max() <= tol * np.abs(b["mol_virial"]).max()
    assert np.abs(a["virial"] - b["virial"]).max() <= tol * np.abs(b["virial"]).max()
    assert np.abs(b["mol_virial"]).max() > 0.0
    rms = np.sqrt((b["forces"] ** 2).sum(1).mean())
    assert np.abs(a["forces"] - b["forces"]).max() <= (1e-12 if pme else 0.0) * rms
