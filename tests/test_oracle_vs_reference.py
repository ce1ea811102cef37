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
