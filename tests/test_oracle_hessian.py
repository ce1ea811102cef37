"""The oracle's restatement of ProtoMol's analytic pair Hessian
(integrators/Hessian.cpp:456-623 with ReducedHessLennardJones,
ReducedHessCoulomb and the C1 / C2 switch Hessians), pinned to ProtoMol's own
Hessian (the compiled reference: Hessian::findForces over a ForceGroup of the
LennardJones and Coulomb forces, then Hessian::evaluate) and against central
differences of the oracle's own forces on the 104-atom vacuum chain, and the
LJ parameter chain rule against differences of the energy (CPU only)."""
import dataclasses

import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import forces as F
from protomol_b200 import systems

FULL = "LennardJones Coulomb -algorithm NonbondedSimpleFull"
FULL_SW = ("LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 -algorithm NonbondedSimpleFull "
           "-switchon 6 -cutoff 9 -cutoff 9")


def forces_of(s, d, pos):
    return oracle.evaluate(s, [F.parse_definition(d)], positions=pos)["forces"]


# the same terms as separate forces, the form Hessian::findForces reads
SEPARATE = {
    FULL: ["LennardJones -algorithm NonbondedSimpleFull", "Coulomb -algorithm NonbondedSimpleFull"],
    FULL_SW: ["LennardJones -switchingFunction C2 -algorithm NonbondedSimpleFull -switchon 6 -cutoff 9",
              "Coulomb -switchingFunction C1 -algorithm NonbondedSimpleFull -cutoff 9"],
}


@pytest.mark.skipif(not oracle.reference_available(), reason="the compiled reference (oracle/_ref) is not built")
@pytest.mark.parametrize("d", [FULL, FULL_SW], ids=["universal", "c2_c1"])
def test_pair_hessian_is_the_reference_hessian(d):
    s = systems.vacuum_chain_104()
    H = oracle.pair_hessian(s, F.parse_definition(d))
    R = oracle.run_reference_hessian(s, [F.parse_definition(x) for x in SEPARATE[d]])
    assert np.abs(H - R).max() <= 1e-12 * np.abs(R).max()


@pytest.mark.parametrize("d", [FULL, FULL_SW], ids=["universal", "c2_c1"])
def test_pair_hessian_matches_force_differences(d):
    s = systems.vacuum_chain_104()
    H = oracle.pair_hessian(s, F.parse_definition(d))
    assert np.allclose(H, H.T, rtol=0, atol=1e-9 * np.abs(H).max())
    rng = np.random.default_rng(2)
    h = 1e-4
    for k in rng.choice(3 * s.n_atoms, 10, replace=False):
        dp = s.positions.copy().reshape(-1)
        dm = dp.copy()
        dp[k] += h
        dm[k] -= h
        col = -(forces_of(s, d, dp.reshape(-1, 3)) - forces_of(s, d, dm.reshape(-1, 3))).reshape(-1) / (2 * h)
        assert np.abs(H[:, k] - col).max() <= 1e-5 * max(1.0, np.abs(col).max()), k


def test_vacuum_chain_has_one_type_per_atom_and_scaled_14():
    s = systems.vacuum_chain_104()
    assert s.n_atoms == 104 and len(set(s.atom_type.tolist())) == 104
    assert (s.exclusions[:, 2] == 1).any() and s.csf == 0.5


def test_lj_parameter_chain_rule_matches_energy_differences():
    """dE/d(eps, Rmin/2) through the table gradient of an analytic model
    (E = sum over a fixed pair list of A r^-12 - B r^-6 with the oracle's
    distances), checked by differences of the parameters."""
    s = systems.vacuum_chain_104()
    rng = np.random.default_rng(5)
    pairs = rng.choice(s.n_atoms, size=(300, 2))
    pairs = pairs[pairs[:, 0] != pairs[:, 1]]
    d = s.positions[pairs[:, 0]] - s.positions[pairs[:, 1]]
    r2 = (d * d).sum(1)

    def energy(tp):
        lj = systems.lj_table_from_types(tp)
        t0, t1 = s.atom_type[pairs[:, 0]], s.atom_type[pairs[:, 1]]
        return float((lj[t0, t1, 0] / r2 ** 6 - lj[t0, t1, 1] / r2 ** 3).sum())

    T = s.n_types
    G = np.zeros((T, T, 4))
    t0, t1 = s.atom_type[pairs[:, 0]], s.atom_type[pairs[:, 1]]
    np.add.at(G, (t0, t1, 0), 0.5 / r2 ** 6)
    np.add.at(G, (t1, t0, 0), 0.5 / r2 ** 6)
    np.add.at(G, (t0, t1, 1), -0.5 / r2 ** 3)
    np.add.at(G, (t1, t0, 1), -0.5 / r2 ** 3)
    grad = F.lj_parameter_gradient(s.type_params, G)
    for t in rng.choice(T, 5, replace=False):
        for col in (0, 1):
            tp_p, tp_m = s.type_params.copy(), s.type_params.copy()
            h = 1e-4 * tp_p[t, col]           # truncation ~1e-8, rounding on E ~ 2e4 negligible
            tp_p[t, col] += h
            tp_m[t, col] -= h
            fd = (energy(tp_p) - energy(tp_m)) / (2 * h)
            assert abs(grad[t, col] - fd) <= 1e-5 * max(1.0, abs(fd)), (t, col, grad[t, col], fd)
