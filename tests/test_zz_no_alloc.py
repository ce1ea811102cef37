"""The allocation-free PME reciprocal entry point (pmgpu_pme_reciprocal_static).

It is for callers that must not allocate GPU memory -- code whose device
memory belongs to another allocator (a framework's caching allocator or a
pool sized to the whole GPU) or that may not call cudaMalloc where the force
is needed.  It runs the kernels of a mixed-precision PME force made with
-reciprocal only, on statically reserved scratch, so its results are checked
against that force evaluated through pmgpu_evaluate_device, with the mixed
tolerances of the other parity tests, on two calls in a row (the second call
finds the scratch as the first one left it).

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from protomol_b200 import _lib
from protomol_b200 import forces as F
from protomol_b200 import systems

MIXED_FORCE_RTOL = 1e-5
MIXED_ENERGY_RTOL = 2e-6

GRID = (24, 24, 24)
ALPHA = 0.35
DEF = ("Coulomb -algorithm PMEwald -reciprocal -interpolation BSpline -gridsize 24 24 24 "
       "-cutoff 9 -order 4 -alpha 0.35")


def _rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def test_sizes_beyond_the_static_scratch_are_rejected():
    lib = _lib.load()
    box = (C.c_double * 3)(24.0, 24.0, 24.0)
    grid = (C.c_int * 3)(*GRID)
    dummy = C.c_void_p(16)   # never dereferenced: the sizes are checked first
    rc = lib.pmgpu_pme_reciprocal_static(0, 65537, dummy, dummy, box, grid, 4, ALPHA, dummy, dummy, 0, None)
    assert rc == 7        # PMGPU_ERR_CAPACITY
    big = (C.c_int * 3)(128, 128, 128)
    rc = lib.pmgpu_pme_reciprocal_static(0, 10, dummy, dummy, box, big, 4, ALPHA, dummy, dummy, 0, None)
    assert rc == 7
    # a prime factor above 7 (22 = 2 x 11) is refused before any launch
    rough = (C.c_int * 3)(22, 24, 24)
    rc = lib.pmgpu_pme_reciprocal_static(0, 10, dummy, dummy, box, rough, 4, ALPHA, dummy, dummy, 0, None)
    assert rc == 5        # PMGPU_ERR_UNSUPPORTED


@pytest.mark.gpu
def test_static_scratch_matches_the_pme_force_on_two_calls():
    import torch
    lib = _lib.load()
    s = systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)
    n = s.n_atoms
    dev = torch.device("cuda:0")
    pos = torch.tensor(s.positions, dtype=torch.float64, device=dev)
    q = torch.tensor(np.asarray(s.scaled_charge, dtype=np.float64), device=dev)

    # the existing entry point: a PME force through the device API
    topo = F.Topology(s, device=0)
    force = F.ForceFactory.make(topo, DEF, "mixed")
    f_ref = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    e_ref = torch.zeros(11, dtype=torch.float64, device=dev)
    arr = (C.c_void_p * 1)(force.handle)
    _lib.check(lib.pmgpu_evaluate_device(topo.handle, 1, arr, C.c_void_p(pos.data_ptr()),
                                         C.c_void_p(f_ref.data_ptr()), C.c_void_p(e_ref.data_ptr()),
                                         _lib.FLAG_VIRIAL), topo.handle)
    _lib.check(lib.pmgpu_synchronize(topo.handle), topo.handle)
    f_ref = f_ref.cpu().numpy()
    e_ref = e_ref.cpu().numpy()
    assert np.abs(f_ref).max() > 0 and e_ref[1] != 0

    box = (C.c_double * 3)(*[float(s.box[k][k]) for k in range(3)])
    grid = (C.c_int * 3)(*GRID)
    for call in range(2):
        f = torch.zeros((n, 3), dtype=torch.float64, device=dev)
        e = torch.zeros(11, dtype=torch.float64, device=dev)
        rc = lib.pmgpu_pme_reciprocal_static(0, n, C.c_void_p(pos.data_ptr()), C.c_void_p(q.data_ptr()), box, grid,
                                             4, ALPHA, C.c_void_p(f.data_ptr()), C.c_void_p(e.data_ptr()),
                                             _lib.FLAG_VIRIAL, None)
        assert rc == 0, f"call {call}: status {rc}"
        f = f.cpu().numpy()
        e = e.cpu().numpy()
        assert _rel_rms(f, f_ref) <= MIXED_FORCE_RTOL, f"call {call}"
        assert abs(e[1] - e_ref[1]) <= MIXED_ENERGY_RTOL * abs(e_ref[1]), f"call {call}"
        vscale = np.abs(e_ref[2:]).max()
        assert np.abs(e[2:] - e_ref[2:]).max() <= MIXED_ENERGY_RTOL * vscale, f"call {call}"
        assert e[0] == 0.0
