"""The Leapfrog integrator on the GPU force path, with positions, velocities
and forces resident in device memory (pmgpu_leapfrog_run).

Mirrors LeapfrogIntegrator (integrators/LeapfrogIntegrator.cpp): ``initialize``
evaluates the forces at the starting positions (initializeForces), ``run(n)``
advances n steps of ``timestep`` fs with one force evaluation per step and
ends with a half kick, so the velocities are synchronous with the positions.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from . import forces as F

_VP = C.c_void_p
BOLTZMANN = 0.001987191         # kcal / mol / K (Constant::BOLTZMANN, base/pmconstants.cpp)


def maxwell_boltzmann(masses: np.ndarray, temperature: float, seed: int) -> np.ndarray:
    """Seeded velocities of a temperature (N x 3, A per internal time unit):
    each component N(0, kT / m), the net momentum removed."""
    m = np.asarray(masses, np.float64)
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(len(m), 3)) * np.sqrt(BOLTZMANN * temperature / m)[:, None]
    v -= (m[:, None] * v).sum(0) / m.sum()
    return v


def kinetic_energy(masses: np.ndarray, velocities: np.ndarray) -> float:
    """0.5 sum m v^2 (kcal/mol), as topologyutilities' kineticEnergy."""
    return float(0.5 * (np.asarray(masses)[:, None] * np.asarray(velocities) ** 2).sum())


class Leapfrog:
    """``constraints`` ({"atoms": (K, 2), "rest": (K,), "shake": (epsilon,
    max_iter) or None, "rattle": (epsilon, max_iter) or None}, the list of
    systems.rattle_shake_constraints) adds ProtoMol's SHAKE post-drift and
    RATTLE post-step modifiers (pmgpu_set_constraints)."""

    def __init__(self, topo: F.Topology, forces: Sequence[F.SystemForce], positions, velocities, masses,
                 timestep: float, device: int = 0, virial: bool = False, constraints=None):
        import torch
        self.topo, self.forces, self.timestep = topo, list(forces), float(timestep)
        self.flags = _lib.FLAG_VIRIAL if virial else 0
        dev = torch.device(f"cuda:{device}")
        self.pos = torch.tensor(np.ascontiguousarray(positions, np.float64), device=dev)
        self.vel = torch.tensor(np.ascontiguousarray(velocities, np.float64), device=dev)
        self.mass = torch.tensor(np.ascontiguousarray(masses, np.float64), device=dev)
        self.force = torch.zeros_like(self.pos)
        self.energy = torch.zeros(11, dtype=torch.float64, device=dev)
        self.masses = np.asarray(masses, np.float64)
        self._arr = (_VP * len(self.forces))(*[f.handle for f in self.forces])
        self.lib = _lib.load()
        c = constraints or {}
        atoms = np.ascontiguousarray(c.get("atoms", np.zeros((0, 2))), np.int32).reshape(-1, 2)
        rest = np.ascontiguousarray(c.get("rest", np.zeros(0)), np.float64)
        shake = c.get("shake") or (0.0, 0)
        rattle = c.get("rattle") or (0.0, 0)
        F.check(self.lib.pmgpu_set_constraints(self.topo.handle, len(rest), atoms.ctypes.data_as(_VP),
                                               rest.ctypes.data_as(_VP), float(shake[0]), int(shake[1]),
                                               float(rattle[0]), int(rattle[1])), self.topo.handle)

    def constraint_limit_hits(self) -> int:
        """Sweeps that stopped at their max_iter (pmgpu_constraint_limit_hits)."""
        return int(self.lib.pmgpu_constraint_limit_hits(self.topo.handle))

    def initialize(self):
        """initializeForces: the forces (and energies) at the starting positions."""
        self.force.zero_()
        self.energy.zero_()
        F.check(self.lib.pmgpu_evaluate_device(self.topo.handle, len(self.forces), self._arr,
                                               _VP(self.pos.data_ptr()), _VP(self.force.data_ptr()),
                                               _VP(self.energy.data_ptr()), self.flags), self.topo.handle)
        return self

    def run(self, n_steps: int):
        F.check(self.lib.pmgpu_leapfrog_run(self.topo.handle, len(self.forces), self._arr, _VP(self.mass.data_ptr()),
                                            _VP(self.pos.data_ptr()), _VP(self.vel.data_ptr()),
                                            _VP(self.force.data_ptr()), _VP(self.energy.data_ptr()),
                                            self.timestep, int(n_steps), self.flags), self.topo.handle)
        return self

    def synchronize(self):
        F.check(self.lib.pmgpu_synchronize(self.topo.handle), self.topo.handle)

    def state(self):
        """(positions, velocities, forces, ScalarStructure) after synchronizing."""
        self.synchronize()
        e = F.ScalarStructure(virial=bool(self.flags & _lib.FLAG_VIRIAL))
        v = self.energy.cpu().numpy()
        e.lennard_jones += float(v[0])
        e.coulomb += float(v[1])
        if self.flags & _lib.FLAG_VIRIAL:
            e.virial_tensor += v[2:11]
        return self.pos.cpu().numpy(), self.vel.cpu().numpy(), self.force.cpu().numpy(), e


class Impulse:
    """ImpulseIntegrator (integrators/ImpulseIntegrator.cpp) over an inner
    Leapfrog, device-resident (pmgpu_impulse_run): the slow forces kick every
    ``cyclelength`` inner steps of ``timestep`` fs, the fast forces drive the
    inner Leapfrog.  ``initialize`` evaluates both groups at the starting
    positions (the integrators' initializeForces)."""

    def __init__(self, topo: F.Topology, slow, fast, positions, velocities, masses, timestep: float,
                 cyclelength: int, device: int = 0, virial: bool = False):
        import torch
        self.topo, self.slow, self.fast = topo, list(slow), list(fast)
        self.timestep, self.cyclelength = float(timestep), int(cyclelength)
        self.flags = _lib.FLAG_VIRIAL if virial else 0
        dev = torch.device(f"cuda:{device}")
        self.pos = torch.tensor(np.ascontiguousarray(positions, np.float64), device=dev)
        self.vel = torch.tensor(np.ascontiguousarray(velocities, np.float64), device=dev)
        self.mass = torch.tensor(np.ascontiguousarray(masses, np.float64), device=dev)
        self.f_slow, self.f_fast = torch.zeros_like(self.pos), torch.zeros_like(self.pos)
        self.e_slow = torch.zeros(11, dtype=torch.float64, device=dev)
        self.e_fast = torch.zeros(11, dtype=torch.float64, device=dev)
        self._slow = (_VP * len(self.slow))(*[f.handle for f in self.slow])
        self._fast = (_VP * len(self.fast))(*[f.handle for f in self.fast])
        self.lib = _lib.load()

    def initialize(self):
        for arr, n, f, e in ((self._slow, len(self.slow), self.f_slow, self.e_slow),
                             (self._fast, len(self.fast), self.f_fast, self.e_fast)):
            f.zero_()
            e.zero_()
            F.check(self.lib.pmgpu_evaluate_device(self.topo.handle, n, arr, _VP(self.pos.data_ptr()),
                                                   _VP(f.data_ptr()), _VP(e.data_ptr()), self.flags), self.topo.handle)
        return self

    def run(self, n_steps: int):
        F.check(self.lib.pmgpu_impulse_run(
            self.topo.handle, len(self.slow), self._slow, len(self.fast), self._fast, _VP(self.mass.data_ptr()),
            _VP(self.pos.data_ptr()), _VP(self.vel.data_ptr()), _VP(self.f_slow.data_ptr()),
            _VP(self.f_fast.data_ptr()), _VP(self.e_slow.data_ptr()), _VP(self.e_fast.data_ptr()),
            self.timestep, self.cyclelength, int(n_steps), self.flags), self.topo.handle)
        return self

    def state(self):
        """(positions, velocities, slow forces, fast forces, total potential energy)."""
        F.check(self.lib.pmgpu_synchronize(self.topo.handle), self.topo.handle)
        es, ef = self.e_slow.cpu().numpy(), self.e_fast.cpu().numpy()
        return (self.pos.cpu().numpy(), self.vel.cpu().numpy(), self.f_slow.cpu().numpy(), self.f_fast.cpu().numpy(),
                float(es[0] + es[1] + ef[0] + ef[1]))
