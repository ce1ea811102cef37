"""Backward pass (pmgpu_adjoint): gradients of the energy w.r.t. the scaled
charges and the LJ table, and the Hessian-vector product of the pair terms,
checked against central finite differences of the forward pass.

The energy is quadratic in the charges and linear in the LJ table entries,
so central differences in those are exact up to rounding (tolerance 1e-7);
the Hessian-vector product is compared with central differences of the
forces at h = 1e-4 A (truncation O(h^2), tolerance 1e-4 relative RMS)."""
import dataclasses

import numpy as np
import pytest

from protomol_b200 import forces as F
from protomol_b200 import systems

pytestmark = pytest.mark.gpu

CUT_EWALD = ("LennardJones CoulombEwaldReal -switchingFunction C2 -switchingFunction Cutoff "
             "-algorithm NonbondedCutoff -switchon 7 -cutoff 9 -alpha 0.35 -cutoff 9 -cutoff 9")
CUT_C2C1 = ("LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 "
            "-algorithm NonbondedCutoff -switchon 7 -cutoff 9 -cutoff 8 -cutoff 9")
PME = ("Coulomb -algorithm PMEwald -reciprocal -correction -interpolation BSpline -gridsize 24 24 24 "
       "-cutoff 9 -alpha 0.35")


def small():
    return systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)


def near_cutoff_atoms(s, rc, band):
    """Atoms with a pair at minimal-image distance within rc +- band."""
    L = np.array([s.box[k][k] for k in range(3)])
    x = s.positions
    mark = np.zeros(s.n_atoms, bool)
    for i in range(s.n_atoms):
        d = x - x[i]
        d -= L * np.rint(d / L)
        r = np.sqrt((d * d).sum(1))
        hit = np.abs(r - rc) < band
        hit[i] = False
        if hit.any():
            mark[i] = True
            mark[hit] = True
    return mark


def forward(s, defs, precision="fp64", positions=None):
    topo = F.Topology(s)
    fs = [F.ForceFactory.make(topo, d, precision) for d in defs]
    out = np.zeros((s.n_atoms, 3))
    e = F.ScalarStructure()
    F.evaluate_group(topo, fs, s.positions if positions is None else positions, out, e)
    return e.lennard_jones + e.coulomb, out


def backward(s, defs, precision="fp64", v=None):
    topo = F.Topology(s)
    fs = [F.ForceFactory.make(topo, d, precision) for d in defs]
    return F.adjoint(topo, fs, s.positions, v)


@pytest.mark.parametrize("defs", [[CUT_EWALD, PME], [CUT_C2C1]], ids=["ewald_pme", "c2_c1"])
def test_charge_gradient_matches_central_differences(defs):
    s = small()
    g = backward(s, defs)["dE_dq"]
    rng = np.random.default_rng(3)
    atoms = list(rng.choice(60, 3, replace=False)) + list(60 + rng.choice(s.n_atoms - 60, 3, replace=False))
    h = 1e-3
    for i in atoms:
        qp, qm = s.scaled_charge.copy(), s.scaled_charge.copy()
        qp[i] += h
        qm[i] -= h
        ep, _ = forward(dataclasses.replace(s, scaled_charge=qp), defs)
        em, _ = forward(dataclasses.replace(s, scaled_charge=qm), defs)
        fd = (ep - em) / (2 * h)
        assert abs(g[i] - fd) <= 1e-7 * max(1.0, abs(fd)), (i, g[i], fd)


def test_lj_table_gradient_matches_central_differences():
    s = small()
    defs = [CUT_C2C1]
    g = backward(s, defs)["dE_dlj"]
    t_water = s.atom_type[-3]            # a water oxygen's type
    t_chain = s.atom_type[5]
    for (t1, t2) in [(t_water, t_water), (t_chain, t_water)]:
        for slot in (0, 1):              # A, B
            lj = s.lj_table.copy()
            h = 1e-6 * abs(lj[t1, t2, slot])
            lp, lm = lj.copy(), lj.copy()
            for tab, sgn in ((lp, 1), (lm, -1)):
                tab[t1, t2, slot] += sgn * h
                if t1 != t2:
                    tab[t2, t1, slot] += sgn * h
            ep, _ = forward(dataclasses.replace(s, lj_table=lp), defs)
            em, _ = forward(dataclasses.replace(s, lj_table=lm), defs)
            fd = (ep - em) / (2 * h)
            an = g[t1, t2, slot] + (g[t2, t1, slot] if t1 != t2 else 0.0)
            assert abs(an - fd) <= 1e-6 * max(1.0, abs(fd)), (t1, t2, slot, an, fd)


@pytest.mark.parametrize("defs", [[CUT_EWALD], [CUT_C2C1]], ids=["ewald", "c2_c1"])
def test_hessian_vector_product_matches_force_differences(defs):
    s = small()
    rng = np.random.default_rng(7)
    v = rng.normal(size=(s.n_atoms, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    hv = backward(s, defs, v=v)["hv"]
    h = 1e-4
    _, fp = forward(s, defs, positions=s.positions + h * v)
    _, fm = forward(s, defs, positions=s.positions - h * v)
    fd = -(fp - fm) / (2 * h)
    # a Cutoff switch makes the force jump where a pair crosses the cutoff:
    # compare the atoms that have no pair within 1e-3 A of it
    keep = ~near_cutoff_atoms(s, 9.0, 1e-3)
    assert keep.sum() > 0.7 * s.n_atoms
    err = np.sqrt(((hv - fd)[keep] ** 2).sum() / (fd[keep] ** 2).sum())
    assert err <= 1e-4, err


def test_mixed_precision_backward_agrees_with_fp64():
    s = small()
    rng = np.random.default_rng(9)
    v = rng.normal(size=(s.n_atoms, 3))
    b64 = backward(s, [CUT_EWALD], "fp64", v=v)
    b32 = backward(s, [CUT_EWALD], "mixed", v=v)
    rel = lambda a, b: np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum())
    assert rel(b32["dE_dq"], b64["dE_dq"]) <= 1e-5
    assert rel(b32["hv"], b64["hv"]) <= 1e-4
    assert rel(b32["dE_dlj"], b64["dE_dlj"]) <= 1e-5


def test_backward_energies_are_the_forward_pair_energies():
    s = small()
    e_fwd, _ = forward(s, [CUT_C2C1])
    b = backward(s, [CUT_C2C1])
    assert abs(b["lennard_jones"] + b["coulomb"] - e_fwd) <= 1e-10 * abs(e_fwd)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("mixed", 1e-4)])
def test_hessian_vector_product_of_pme_matches_oracle_force_differences(precision, tol):
    """The reciprocal and correction terms (smooth: no cutoff) against
    central differences of the oracle's FP64 PME forces, h = 1e-4 A."""
    from oracle import oracle
    s = small()
    rng = np.random.default_rng(17)
    v = rng.normal(size=(s.n_atoms, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    hv = backward(s, [PME], precision, v=v)["hv"]
    h = 1e-4
    spec = [F.parse_definition(PME)]
    fp = oracle.evaluate(s, spec, positions=s.positions + h * v)["forces"]
    fm = oracle.evaluate(s, spec, positions=s.positions - h * v)["forces"]
    fd = -(fp - fm) / (2 * h)
    err = np.sqrt(((hv - fd) ** 2).sum() / (fd ** 2).sum())
    print(f"\nPME H v ({precision}) against oracle differences: {err:.2e}")
    assert err <= tol, err


def test_hessian_vector_product_of_split_pme_matches_force_differences():
    """Ewald real space as a cutoff force plus PME reciprocal + correction,
    FP64, against central differences of the GPU forces."""
    s = small()
    rng = np.random.default_rng(23)
    v = rng.normal(size=(s.n_atoms, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    defs = [CUT_EWALD, PME]
    hv = backward(s, defs, v=v)["hv"]
    h = 1e-4
    _, fp = forward(s, defs, positions=s.positions + h * v)
    _, fm = forward(s, defs, positions=s.positions - h * v)
    fd = -(fp - fm) / (2 * h)
    keep = ~near_cutoff_atoms(s, 9.0, 1e-3)
    err = np.sqrt(((hv - fd)[keep] ** 2).sum() / (fd[keep] ** 2).sum())
    assert err <= 1e-4, err
