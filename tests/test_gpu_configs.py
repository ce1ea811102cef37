"""Configuration-level parity of the GPU forces against the oracle.

* The batched-water configuration (96 boxes of 100-3,000 TIP3P waters,
  cutoff 9 with C2 8 -> 9, Ewald real space + PME on a ~1 A grid): its
  largest box and a box under 18 A (below twice the cutoff, where the pair
  force keeps the reference's single minimal image per cell pair), each
  evaluated alone in mixed precision, against the oracle at 1e-7 of the
  total energy and of the virial.
* A non-neutral box: PME's charged-system term (a constant energy and a
  virial diagonal, forces/NonbondedPMEwaldSystemForce.h:604-628), FP64 and
  mixed, against the oracle (which the compiled reference pins, see
  tests/test_oracle_vs_reference.py).
* The charge gradient of the 14,281-atom cutoff + PME energy on 64 atoms
  (chain and water, spread over the box) against central differences of the
  FP64 energies, the charges changed in place on one system.
"""
import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import forces as F
from protomol_b200 import systems, workloads

pytestmark = pytest.mark.gpu

FORCE_RTOL = 1e-5
METRIC_ENERGY_RTOL = 1e-7
COULOMB_ONLY_VIRIAL_RTOL = 2e-6


def _eval(s, defs, precision):
    topo = F.Topology(s)
    fs = [F.ForceFactory.make(topo, d, precision) for d in defs]
    out = np.zeros((s.n_atoms, 3))
    e = F.ScalarStructure(virial=True)
    F.evaluate_group(topo, fs, s.positions, out, e)
    return topo, out, e


def _rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def _batched_box(which):
    ws = workloads.batched96()
    sizes = [w.system.n_atoms for w in ws]
    if which == "largest":
        return ws[int(np.argmax(sizes))]
    small = [w for w in ws if w.system.box_lengths.min() < 18.0]
    return min(small, key=lambda w: w.system.n_atoms)


@pytest.mark.parametrize("which", ["largest", "under_18A"])
def test_batched_water_boxes_against_oracle(which):
    w = _batched_box(which)
    s = w.system
    ref = oracle.evaluate(s, [F.parse_definition(d) for d in w.forces])
    topo, f, e = _eval(s, w.forces, "mixed")
    etot, rtot = e.lennard_jones + e.coulomb, ref["lennard_jones"] + ref["coulomb"]
    de = abs(etot - rtot) / abs(rtot)
    dv = np.linalg.norm(e.virial_tensor - ref["virial"]) / np.linalg.norm(ref["virial"])
    err = _rel_rms(f, ref["forces"])
    print(f"\n{which}: {s.n_atoms} atoms, L {s.box_lengths[0]:.2f} A, layout {topo.pair_layout()}: "
          f"force {err:.2e} energy {de:.2e} virial {dv:.2e}")
    assert topo.pair_layout() == ("columns" if which == "largest" else "cells")
    assert err <= FORCE_RTOL
    assert de <= METRIC_ENERGY_RTOL
    assert dv <= METRIC_ENERGY_RTOL


def charged_chain():
    s = systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)
    s.scaled_charge = s.scaled_charge.copy()
    s.scaled_charge[5] += 0.5 * systems.SQRT_COULOMB_CONSTANT
    return s


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_charged_system_pme_against_oracle(precision):
    s = charged_chain()
    assert abs(s.scaled_charge.sum() * 0.00268283) > 1e-5
    defs = ["Coulomb -algorithm PMEwald -real -reciprocal -correction -interpolation BSpline "
            "-gridsize 24 24 24 -cutoff 9 -alpha 0.35"]
    ref = oracle.evaluate(s, [F.parse_definition(d) for d in defs])
    _, f, e = _eval(s, defs, precision)
    if precision == "fp64":
        rms = np.sqrt((ref["forces"] ** 2).sum(1).mean())
        assert np.abs(f - ref["forces"]).max() <= 1e-9 * rms
        assert abs(e.coulomb - ref["coulomb"]) <= 1e-10 * abs(ref["coulomb"])
        assert np.abs(e.virial_tensor - ref["virial"]).max() <= 1e-10 * np.abs(ref["virial"]).max()
    else:
        assert _rel_rms(f, ref["forces"]) <= FORCE_RTOL
        assert abs(e.coulomb - ref["coulomb"]) <= METRIC_ENERGY_RTOL * abs(ref["coulomb"])
        # a Coulomb-only virial is a near cancellation of pair terms led by the
        # FP32 forces of hydrogen-bonded pairs (4.4e-7 measured)
        assert np.linalg.norm(e.virial_tensor - ref["virial"]) <= COULOMB_ONLY_VIRIAL_RTOL * np.linalg.norm(ref["virial"])
    # the oracle's result holds the charged-system term, -pi (sum q~)^2 /
    # (2 V alpha^2), on the energy and on each virial diagonal entry
    V = float(np.prod(s.box_lengths))
    alpha = ref["alpha"]
    term = -np.pi / (2 * V * alpha ** 2) * s.scaled_charge.sum() ** 2
    assert ref["e_charged"] == pytest.approx(term, rel=1e-12) and term < -0.05


def test_charge_gradient_of_the_14281_atom_pme_box_on_64_atoms(chain14281):
    s = chain14281
    w = workloads.chain14281()
    topo = F.Topology(s)
    fs = [F.ForceFactory.make(topo, d, "fp64") for d in w.forces]
    g = F.adjoint(topo, fs, s.positions)["dE_dq"]
    rng = np.random.default_rng(64)
    atoms = np.concatenate([rng.choice(892, 16, replace=False),
                            892 + rng.choice(s.n_atoms - 892, 48, replace=False)])
    h = 1e-3 * systems.SQRT_COULOMB_CONSTANT
    out = np.zeros((s.n_atoms, 3))
    worst = 0.0
    for i in atoms:
        es = []
        for sign in (1, -1):
            q = s.scaled_charge.copy()
            q[i] += sign * h
            s2 = s.copy()
            s2.scaled_charge = q
            topo.set_topology(s2)                # the same system and forces, new charges
            e = F.ScalarStructure()
            F.evaluate_group(topo, fs, s.positions, out, e)
            es.append(e.potential_energy())
        fd = (es[0] - es[1]) / (2 * h)
        worst = max(worst, abs(g[i] - fd) / max(1.0, abs(fd)))
        assert abs(g[i] - fd) <= 1e-6 * max(1.0, abs(fd)), (int(i), g[i], fd)
    print(f"\n64-atom PME charge gradient: worst relative error {worst:.2e}")
