"""Differentiation on the GPU, the adjoint configuration:

part one -- the 104-atom vacuum chain with all-pairs LennardJones + Coulomb
(NonbondedSimpleFull, 1-2 / 1-3 excluded, 1-4 scaled 0.5): the forward
all-pairs force against the oracle, 64 seeded unit-vector Hessian-vector
products in FP64 and FP32 against ProtoMol's analytic Hessian (the oracle's
restatement of integrators/Hessian.cpp, pinned in test_oracle_hessian.py) and
against central differences of the forces (h = 1e-4 A), and the gradients
w.r.t. charges (h = 1e-3 e) and LJ eps / Rmin/2 against central differences;

part two -- the same gradients on the 14,281-atom cutoff + PME box.

Tolerances: FP64 Hessian-vector products 1e-10 relative RMS of the oracle's;
FP32 ones 1e-4 (single-precision pair math); finite differences 1e-4
(truncation O(h^2)); charge differences 1e-6: the energy is quadratic in the
charges, so a central difference is exact at any step and the step is taken
large enough that the rounding of a ~1e4 kcal/mol total stays below it."""
import dataclasses

import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import forces as F
from protomol_b200 import systems, workloads

pytestmark = pytest.mark.gpu

FULL = "LennardJones Coulomb -algorithm NonbondedSimpleFull"
SQRT_K = 18.2226123264                     # charge scale: q~ = q sqrt(332.0636)


def rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def evaluate(s, defs, precision="fp64", positions=None):
    topo = F.Topology(s)
    fs = [F.ForceFactory.make(topo, d, precision) for d in defs]
    out = np.zeros((s.n_atoms, 3))
    e = F.ScalarStructure()
    F.evaluate_group(topo, fs, s.positions if positions is None else positions, out, e)
    return e, out


def backward(s, defs, precision="fp64", v=None):
    topo = F.Topology(s)
    fs = [F.ForceFactory.make(topo, d, precision) for d in defs]
    return F.adjoint(topo, fs, s.positions, v)


@pytest.fixture(scope="module")
def chain():
    return systems.vacuum_chain_104()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_vacuum_all_pairs_forward_matches_oracle(chain, precision):
    ref = oracle.evaluate(chain, [F.parse_definition(FULL)])
    e, f = evaluate(chain, [FULL], precision)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rel(f, ref["forces"]) <= tol
    scale = abs(ref["lennard_jones"]) + abs(ref["coulomb"])
    etol = 1e-12 if precision == "fp64" else 2e-6
    assert abs(e.lennard_jones - ref["lennard_jones"]) <= etol * scale
    assert abs(e.coulomb - ref["coulomb"]) <= etol * scale
    assert np.abs(e.virial_tensor - ref["virial"]).max() <= 10 * etol * np.abs(ref["virial"]).max()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-4)])
def test_64_hessian_vector_products_match_the_reference_hessian(chain, precision, tol):
    H = oracle.pair_hessian(chain, F.parse_definition(FULL))
    rng = np.random.default_rng(64)
    topo = F.Topology(chain)
    fs = [F.ForceFactory.make(topo, FULL, precision)]
    worst = 0.0
    for _ in range(64):
        v = rng.normal(size=3 * chain.n_atoms)
        v /= np.linalg.norm(v)
        hv = F.adjoint(topo, fs, chain.positions, v.reshape(-1, 3))["hv"].reshape(-1)
        worst = max(worst, rel(hv, H @ v))
    assert worst <= tol, worst


def test_hessian_vector_products_match_force_differences(chain):
    rng = np.random.default_rng(65)
    h = 1e-4
    for _ in range(4):
        v = rng.normal(size=(chain.n_atoms, 3))
        v /= np.linalg.norm(v)
        hv = backward(chain, [FULL], v=v)["hv"]
        _, fp = evaluate(chain, [FULL], positions=chain.positions + h * v)
        _, fm = evaluate(chain, [FULL], positions=chain.positions - h * v)
        assert rel(hv, -(fp - fm) / (2 * h)) <= 1e-4


def _param_fd(s, defs, t, col, h):
    tp_p, tp_m = s.type_params.copy(), s.type_params.copy()
    tp_p[t, col] += h
    tp_m[t, col] -= h
    sp = dataclasses.replace(s, type_params=tp_p, lj_table=systems.lj_table_from_types(tp_p))
    sm = dataclasses.replace(s, type_params=tp_m, lj_table=systems.lj_table_from_types(tp_m))
    ep, _ = evaluate(sp, defs)
    em, _ = evaluate(sm, defs)
    return (ep.potential_energy() - em.potential_energy()) / (2 * h)


def _check_gradients(s, defs, atoms, precision="fp64"):
    b = backward(s, defs, precision)
    g_par = F.lj_parameter_gradient(s.type_params, b["dE_dlj"])
    h = 1e-3 * SQRT_K                      # 1e-3 e
    for i in atoms:
        qp, qm = s.scaled_charge.copy(), s.scaled_charge.copy()
        qp[i] += h
        qm[i] -= h
        ep, _ = evaluate(dataclasses.replace(s, scaled_charge=qp), defs)
        em, _ = evaluate(dataclasses.replace(s, scaled_charge=qm), defs)
        fd = (ep.potential_energy() - em.potential_energy()) / (2 * h)
        assert abs(b["dE_dq"][i] - fd) <= 1e-6 * max(1.0, abs(fd)), ("charge", i, b["dE_dq"][i], fd)
        t = s.atom_type[i]
        for col in (0, 1):                 # eps, Rmin/2 (types with eps = 0 have no LJ term)
            if s.type_params[t, 0] == 0.0:
                continue
            hp = 1e-4 * s.type_params[t, col]
            fd = _param_fd(s, defs, t, col, hp)
            assert abs(g_par[t, col] - fd) <= 1e-5 * max(1.0, abs(fd)), ("lj", i, col, g_par[t, col], fd)
    return b


def test_charge_and_lj_gradients_on_the_vacuum_chain(chain):
    b64 = _check_gradients(chain, [FULL], [0, 17, 51, 103])
    b32 = backward(chain, [FULL], "mixed")
    assert rel(b32["dE_dq"], b64["dE_dq"]) <= 1e-5
    assert rel(b32["dE_dlj"], b64["dE_dlj"]) <= 1e-5


def test_charge_and_lj_gradients_on_the_14281_atom_pme_box(chain14281):
    w = workloads.chain14281()
    # chain atoms (own LJ types) and a water
    oxygen = 892 + 3 * 1369                # a water oxygen (waters follow the 892 chain atoms)
    assert chain14281.type_params[chain14281.atom_type[oxygen], 0] > 0
    _check_gradients(chain14281, w.forces, [3, 400, 891, oxygen])


# ---------------------------------------------------------------- autograd
# The forward/backward pair as a torch.autograd.Function, for the test
# harness only: E(x, q~) forward through pmgpu_evaluate; its backward is -F
# and dE/dq~ (pmgpu_adjoint).  The position gradient is itself a Function
# whose backward is the adjoint's Hessian-vector product, so double backward
# (torch.autograd.functional.vhp; H is symmetric, v^T H = (H v)^T) runs on
# the GPU kernels as well.

class _Graph:
    """Topology + forces of one system, rebuilt when the charges change."""

    def __init__(self, s, defs, precision="fp64"):
        self.s, self.defs, self.precision = s, defs, precision
        self.key = None

    def forces_for(self, q):
        key = q.tobytes()
        if key != self.key:
            self.topo = F.Topology(dataclasses.replace(self.s, scaled_charge=q.copy()))
            self.fs = [F.ForceFactory.make(self.topo, d, self.precision) for d in self.defs]
            self.key = key
        return self.topo, self.fs


def _energy_fn(graph):
    import torch

    class GradFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x, q):
            topo, fs = graph.forces_for(q.detach().numpy())
            out = np.zeros((topo.n_atoms, 3))
            F.evaluate_group(topo, fs, x.detach().numpy(), out, F.ScalarStructure())
            ctx.save_for_backward(x, q)
            return torch.from_numpy(-out)                 # dE/dx = -F

        @staticmethod
        def backward(ctx, v):
            x, q = ctx.saved_tensors
            topo, fs = graph.forces_for(q.detach().numpy())
            hv = F.adjoint(topo, fs, x.detach().numpy(), v.detach().numpy())["hv"]
            return torch.from_numpy(hv), None

    class EnergyFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x, q):
            topo, fs = graph.forces_for(q.detach().numpy())
            e = F.ScalarStructure()
            F.evaluate_group(topo, fs, x.detach().numpy(), np.zeros((topo.n_atoms, 3)), e)
            ctx.save_for_backward(x, q)
            return torch.tensor(e.potential_energy(), dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            x, q = ctx.saved_tensors
            topo, fs = graph.forces_for(q.detach().numpy())
            dq = F.adjoint(topo, fs, x.detach().numpy())["dE_dq"]
            return g * GradFn.apply(x, q), g * torch.from_numpy(dq)

    return EnergyFn.apply


def test_autograd_gradients_pass_gradcheck(chain):
    import torch
    energy = _energy_fn(_Graph(chain, [FULL]))
    x = torch.tensor(chain.positions, dtype=torch.float64, requires_grad=True)
    q = torch.tensor(chain.scaled_charge, dtype=torch.float64, requires_grad=True)
    # central differences of E against -F and dE/dq~ (step 1e-4 A / 1e-4 e~:
    # truncation O(h^2) in x, exact in the quadratic q~)
    assert torch.autograd.gradcheck(energy, (x, q), eps=1e-4, atol=1e-5, rtol=1e-4)


def test_autograd_double_backward_is_the_reference_hessian(chain):
    import torch
    energy = _energy_fn(_Graph(chain, [FULL]))
    q = torch.tensor(chain.scaled_charge, dtype=torch.float64)
    H = oracle.pair_hessian(chain, F.parse_definition(FULL))
    rng = np.random.default_rng(66)
    x = torch.tensor(chain.positions, dtype=torch.float64)
    for _ in range(4):
        v = rng.normal(size=(chain.n_atoms, 3))
        v /= np.linalg.norm(v)
        _, hv = torch.autograd.functional.vhp(lambda xx: energy(xx, q), x, torch.from_numpy(v))
        assert rel(hv.numpy().reshape(-1), H @ v.reshape(-1)) <= 1e-10


def test_autograd_charge_gradient_on_the_14281_atom_pme_box(chain14281):
    import torch
    w = workloads.chain14281()
    energy = _energy_fn(_Graph(chain14281, w.forces, "mixed"))
    x = torch.tensor(chain14281.positions, dtype=torch.float64)
    q = torch.tensor(chain14281.scaled_charge, dtype=torch.float64, requires_grad=True)
    (gq,) = torch.autograd.grad(energy(x, q), q)
    topo = F.Topology(chain14281)
    fs = [F.ForceFactory.make(topo, d, "fp64") for d in w.forces]
    ref = F.adjoint(topo, fs, chain14281.positions)["dE_dq"]
    assert rel(gq.numpy(), ref) <= 1e-5               # mixed against the FP64 backward pass


# ---------------------------------------------------------------- dense Hessian
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_dense_hessian_is_the_reference_hessian(chain, precision, tol):
    H = oracle.pair_hessian(chain, F.parse_definition(FULL))
    topo = F.Topology(chain)
    fs = [F.ForceFactory.make(topo, FULL, precision)]
    Hg = F.hessian(topo, fs, chain.positions)
    assert rel(Hg, H) <= tol
    assert np.abs(Hg - Hg.T).max() <= 10 * tol * np.abs(H).max()
    v = np.random.default_rng(67).normal(size=(chain.n_atoms, 3))
    hv = F.adjoint(topo, fs, chain.positions, v)["hv"].reshape(-1)
    assert rel(Hg @ v.reshape(-1), hv) <= tol                 # the same blocks as the HVP


def test_dense_hessian_of_a_periodic_cutoff_force():
    """The minimal image and the cutoff: a 1,260-atom chain in water with LJ
    C2 + Coulomb C1 (cutoff 9), against the oracle's periodic Hessian."""
    s = systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)
    d = ("LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 -algorithm NonbondedCutoff "
         "-switchon 7 -cutoff 9 -cutoff 9 -cutoff 9")
    H = oracle.pair_hessian(s, F.parse_definition(d))
    topo = F.Topology(s)
    Hg = F.hessian(topo, [F.ForceFactory.make(topo, d, "fp64")], s.positions)
    assert rel(Hg, H) <= 1e-10
