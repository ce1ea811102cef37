"""ctypes binding of libpmgpu.so (include/pmgpu.h).

Loading fails loudly: there is no CPU fallback for any force.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpmgpu.so")

PMGPU_OK = 0
ERRORS = {1: "PMGPU_ERR_ARG", 2: "PMGPU_ERR_CUDA", 3: "PMGPU_ERR_OVERFLOW", 4: "PMGPU_ERR_STATE",
          5: "PMGPU_ERR_UNSUPPORTED", 6: "PMGPU_ERR_NOMEM", 7: "PMGPU_ERR_CAPACITY"}

POT = {"LennardJones": 1, "Coulomb": 2, "CoulombEwaldReal": 3,
       "LennardJonesTable": 4, "CoulombTable": 5, "CoulombEwaldRealTable": 6}
SW = {"Universal": 0, "Cutoff": 1, "C1": 2, "C2": 3, "Shift": 4}
PRECISION = {"mixed": 0, "fp64": 1}
FLAG_VIRIAL = 1
FLAG_MOLECULAR_VIRIAL = 2

# every symbol include/pmgpu.h declares
EXPORTS = [
    "pmgpu_system_create", "pmgpu_system_destroy", "pmgpu_set_topology", "pmgpu_set_box",
    "pmgpu_cutoff_create", "pmgpu_pme_create", "pmgpu_force_destroy", "pmgpu_pme_alpha",
    "pmgpu_evaluate", "pmgpu_evaluate_device", "pmgpu_synchronize", "pmgpu_stream",
    "pmgpu_launch_count", "pmgpu_last_error", "pmgpu_get_cells", "pmgpu_get_pairs", "pmgpu_pair_layout",
    "pmgpu_set_pair_list", "pmgpu_pair_list_builds", "pmgpu_set_molecule_positions",
    "pmgpu_set_profiling", "pmgpu_phase_times", "pmgpu_pme_reciprocal_static",
    "pmgpu_batch_create", "pmgpu_batch_destroy", "pmgpu_batch_add", "pmgpu_batch_evaluate",
    "pmgpu_batch_synchronize", "pmgpu_batch_last_error", "pmgpu_batch_stream", "pmgpu_batch_set_pair_launch",
    "pmgpu_adjoint",
    "pmgpu_full_create", "pmgpu_lookup_table", "pmgpu_get_tuning", "pmgpu_set_tuning", "pmgpu_autotune", "pmgpu_batch_autotune",
    "pmgpu_leapfrog_run", "pmgpu_hessian", "pmgpu_impulse_run", "pmgpu_set_constraints",
    "pmgpu_constraint_limit_hits",
]
PHASES = ["bin", "pair", "pme_correction", "pme_spread", "pme_fft", "pme_gather", "finalize", "pair_list",
          "pme_energy64"]


class CutoffParams(C.Structure):
    _fields_ = [
        ("n_terms", C.c_int), ("pot", C.c_int * 2), ("sw", C.c_int * 2),
        ("switchon", C.c_double * 2), ("cutoff", C.c_double * 2), ("alpha", C.c_double * 2),
        ("algorithm_cutoff", C.c_double), ("precision", C.c_int),
    ]


class PmeParams(C.Structure):
    _fields_ = [
        ("real", C.c_int), ("reciprocal", C.c_int), ("correction", C.c_int),
        ("grid", C.c_int * 3), ("order", C.c_int), ("cutoff", C.c_double),
        ("accuracy", C.c_double), ("alpha", C.c_double), ("precision", C.c_int),
    ]


class Tuning(C.Structure):
    _fields_ = [("chunk_entries", C.c_int), ("pair_blocks_per_sm", C.c_int), ("fft_lines", C.c_int),
                ("pme_concurrent", C.c_int), ("fp64_pairs", C.c_int), ("ms_per_eval", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Energies(C.Structure):
    _fields_ = [("lennard_jones", C.c_double), ("coulomb", C.c_double), ("virial", C.c_double * 9)]


class EnergiesMol(C.Structure):
    """pmgpu_energies_mol: the pmgpu_energies slots and the molecular virial."""
    _fields_ = [("lennard_jones", C.c_double), ("coulomb", C.c_double), ("virial", C.c_double * 9),
                ("molecular_virial", C.c_double * 9)]


class PmgpuError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


_lib = None


def load():
    """Loads the in-tree libpmgpu.so; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m protomol_b200.build` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    lib.pmgpu_system_create.argtypes = [C.c_int, C.POINTER(vp)]
    lib.pmgpu_system_destroy.argtypes = [vp]
    lib.pmgpu_set_topology.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int, vp, C.c_int, vp, vp, vp, C.c_double]
    lib.pmgpu_set_box.argtypes = [vp, dp, dp, dp, dp, C.c_double]
    lib.pmgpu_cutoff_create.argtypes = [vp, C.POINTER(CutoffParams), C.POINTER(vp)]
    lib.pmgpu_pme_create.argtypes = [vp, C.POINTER(PmeParams), C.POINTER(vp)]
    lib.pmgpu_force_destroy.argtypes = [vp]
    lib.pmgpu_pme_alpha.argtypes = [vp, dp]
    lib.pmgpu_evaluate.argtypes = [vp, C.c_int, C.POINTER(vp), vp, vp, vp, C.c_uint]
    lib.pmgpu_set_molecule_positions.argtypes = [vp, C.c_int, vp]
    lib.pmgpu_evaluate_device.argtypes = [vp, C.c_int, C.POINTER(vp), vp, vp, vp, C.c_uint]
    lib.pmgpu_synchronize.argtypes = [vp]
    lib.pmgpu_stream.argtypes = [vp]
    lib.pmgpu_stream.restype = vp
    lib.pmgpu_launch_count.argtypes = [vp]
    lib.pmgpu_launch_count.restype = C.c_longlong
    lib.pmgpu_last_error.argtypes = [vp, C.c_char_p, C.c_int]
    lib.pmgpu_get_cells.argtypes = [vp, vp, vp]
    lib.pmgpu_pair_layout.argtypes = [vp]
    lib.pmgpu_set_pair_list.argtypes = [vp, C.c_double, C.c_int]
    lib.pmgpu_pair_list_builds.argtypes = [vp]
    lib.pmgpu_pair_list_builds.restype = C.c_longlong
    lib.pmgpu_get_pairs.argtypes = [vp, vp, vp, C.POINTER(C.c_longlong), vp, C.c_longlong]
    lib.pmgpu_set_profiling.argtypes = [vp, C.c_int]
    lib.pmgpu_phase_times.argtypes = [vp, vp, C.c_int, C.POINTER(C.c_longlong)]
    lib.pmgpu_pme_reciprocal_static.argtypes = [C.c_int, C.c_int, vp, vp, dp, ip, C.c_int, C.c_double,
                                                vp, vp, C.c_uint, vp]
    lib.pmgpu_batch_create.argtypes = [C.c_int, C.POINTER(vp)]
    lib.pmgpu_batch_destroy.argtypes = [vp]
    lib.pmgpu_batch_add.argtypes = [vp, vp, C.c_int, vp, vp, vp, vp, C.c_uint]
    lib.pmgpu_batch_evaluate.argtypes = [vp]
    lib.pmgpu_batch_set_pair_launch.argtypes = [vp, C.c_int]
    lib.pmgpu_batch_synchronize.argtypes = [vp]
    lib.pmgpu_batch_last_error.argtypes = [vp, C.c_char_p, C.c_int]
    lib.pmgpu_batch_stream.argtypes = [vp]
    lib.pmgpu_batch_stream.restype = vp
    lib.pmgpu_adjoint.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp]
    lib.pmgpu_full_create.argtypes = [vp, C.POINTER(CutoffParams), C.POINTER(vp)]
    lib.pmgpu_lookup_table.restype = C.c_longlong
    lib.pmgpu_lookup_table.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, vp, C.c_longlong]
    lib.pmgpu_get_tuning.argtypes = [vp, C.POINTER(Tuning)]
    lib.pmgpu_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
    lib.pmgpu_autotune.argtypes = [vp, C.c_int, C.POINTER(vp), vp, C.c_uint, C.c_int, C.POINTER(Tuning)]
    lib.pmgpu_batch_autotune.argtypes = [vp, C.c_int, C.POINTER(Tuning)]
    lib.pmgpu_hessian.argtypes = [vp, C.c_int, C.POINTER(vp), vp, vp]
    lib.pmgpu_impulse_run.argtypes = [vp, C.c_int, C.POINTER(vp), C.c_int, C.POINTER(vp), vp, vp, vp, vp, vp, vp, vp,
                                      C.c_double, C.c_int, C.c_int, C.c_uint]
    lib.pmgpu_leapfrog_run.argtypes = [vp, C.c_int, C.POINTER(vp), vp, vp, vp, vp, vp, C.c_double, C.c_int,
                                       C.c_uint]
    lib.pmgpu_set_constraints.argtypes = [vp, C.c_int, vp, vp, C.c_double, C.c_int, C.c_double, C.c_int]
    lib.pmgpu_constraint_limit_hits.argtypes = [vp]
    lib.pmgpu_constraint_limit_hits.restype = C.c_longlong
    _lib = lib
    return lib


def last_error(sys_handle) -> str:
    buf = C.create_string_buffer(1024)
    load().pmgpu_last_error(sys_handle, buf, 1024)
    return buf.value.decode(errors="replace")


def check(code, sys_handle=None):
    if code != PMGPU_OK:
        raise PmgpuError(code, last_error(sys_handle) if sys_handle else "")
