"""Batches of independent systems (the 96 uneven water boxes of the batched
configuration): one CUDA graph launch evaluates every member, and across GPUs
the members are sharded by atom count with no collective.

The reference evaluates one system per process (ForceGroup::
evaluateSystemForces, forces/ForceGroup.cpp:70-82); a batch is that call for
many systems at once, each member's results identical to evaluating it alone.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from . import _lib
from . import forces as F

_VP = C.c_void_p


def shard_by_atoms(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Greedy longest-first partition of the systems over `world` ranks:
    each system, largest first, goes to the rank with the fewest atoms so far
    (ties to the lower rank).  Deterministic, so every rank computes the same
    assignment without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for k in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += int(sizes[k])
    return [sorted(v) for v in out]


class Batch:
    """Members = (Topology, forces, positions); device buffers are owned here.

    ``evaluate()`` launches every member's evaluation with one graph launch;
    ``results()`` returns per-member (forces N x 3, ScalarStructure)."""

    def __init__(self, device: int = 0):
        import torch
        self._torch = torch
        self.device = device
        self.lib = _lib.load()
        h = _VP()
        _lib.check(self.lib.pmgpu_batch_create(device, C.byref(h)))
        self.handle = h
        self.members = []

    def add(self, topo: F.Topology, forces: Sequence[F.SystemForce], positions: np.ndarray,
            virial: bool = True):
        torch = self._torch
        dev = torch.device(f"cuda:{self.device}")
        pos = torch.tensor(np.ascontiguousarray(positions, np.float64), device=dev)
        fout = torch.zeros_like(pos)
        energy = torch.zeros(11, dtype=torch.float64, device=dev)
        arr = (_VP * len(forces))(*[f.handle for f in forces])
        flags = _lib.FLAG_VIRIAL if virial else 0
        rc = self.lib.pmgpu_batch_add(self.handle, topo.handle, len(forces), arr, _VP(pos.data_ptr()),
                                      _VP(fout.data_ptr()), _VP(energy.data_ptr()), flags)
        self._check(rc)
        self.members.append((topo, list(forces), pos, fout, energy, virial))

    def _check(self, rc):
        if rc != _lib.PMGPU_OK:
            buf = C.create_string_buffer(1024)
            self.lib.pmgpu_batch_last_error(self.handle, buf, 1024)
            raise _lib.PmgpuError(rc, buf.value.decode(errors="replace"))

    @property
    def stream(self) -> int:
        return int(self.lib.pmgpu_batch_stream(self.handle) or 0)

    def zero(self):
        for _, _, _, fout, energy, _ in self.members:
            fout.zero_()
            energy.zero_()

    def evaluate(self):
        self._check(self.lib.pmgpu_batch_evaluate(self.handle))

    def set_pair_launch(self, one_launch: bool):
        """pmgpu_batch_set_pair_launch: the members' column-path pair kernels
        as one persistent launch (True, the default) or one per member."""
        self._check(self.lib.pmgpu_batch_set_pair_launch(self.handle, 1 if one_launch else 0))

    def autotune(self, evals: int = 5) -> dict:
        """pmgpu_batch_autotune: one tuning for every member, timed as whole
        batch launches; the members' outputs are zeroed afterwards."""
        t = _lib.Tuning()
        self._check(self.lib.pmgpu_batch_autotune(self.handle, int(evals), C.byref(t)))
        self.zero()
        return t.as_dict()

    def synchronize(self):
        self._check(self.lib.pmgpu_batch_synchronize(self.handle))

    def results(self):
        self.synchronize()
        out = []
        for _, _, _, fout, energy, virial in self.members:
            e = F.ScalarStructure(virial=virial)
            v = energy.cpu().numpy()
            e.lennard_jones += float(v[0])
            e.coulomb += float(v[1])
            if virial:
                e.virial_tensor += v[2:11]
            out.append((fout.cpu().numpy(), e))
        return out

    def close(self):
        if getattr(self, "handle", None):
            self.lib.pmgpu_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
