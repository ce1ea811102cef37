"""CPU checks of the drop-in boundary: libpmgpu.so loads, exports exactly
what include/pmgpu.h declares, refuses to run without a GPU, and the
force-definition parser follows ForceFactory's keyword rules."""
import ctypes as C
import os
import re
import subprocess

import pytest

from protomol_b200 import _lib
from protomol_b200 import forces as F

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pmgpu.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(pmgpu_[a-z_]+)\s*\(", text)))


def test_header_declares_what_the_binding_uses():
    assert declared_symbols() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    for name in declared_symbols():
        assert name in exported, name
        assert getattr(lib, name) is not None


def test_no_gpu_means_an_error_not_a_fallback():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = C.c_void_p()
    assert _lib.load().pmgpu_system_create(0, C.byref(h)) == 2   # PMGPU_ERR_CUDA
    assert not h.value


def test_parse_split_form_of_the_bpti_conf():
    # the force line of examples/bpti_water_14281/bpti.pme.opt.conf, reordered
    d = F.parse_definition("force LennardJones CoulombEwaldReal -algorithm NonbondedCutoff "
                           "-switchingFunction C2 -switchingFunction Cutoff "
                           "-switchon 8 -cutoff 10 -alpha 0.3 -cutoff 10 -cutoff 10")
    assert d == {"kind": "cut", "algo_cutoff": 10.0,
                 "terms": [("C2", "LennardJones", 8.0, 10.0, 0.0), ("Cutoff", "CoulombEwaldReal", 0.0, 10.0, 0.3)]}


def test_parse_pme_defaults_and_positional_gridsize():
    d = F.parse_definition("Coulomb -algorithm PMEwald -reciprocal -correction -interpolation BSpline "
                           "-gridsize 60 48 48 -cutoff 10")
    assert d["grid"] == (60, 48, 48) and d["order"] == 4 and d["accuracy"] == 1e-6 and d["alpha"] == -1.0
    assert d["reciprocal"] == 1 and d["correction"] == 1 and d["real"] == 0


def test_parse_cutoff_keywords_match_left_to_right():
    # getParameters order: C2 (-switchon, -cutoff), C1 (-cutoff), algorithm -cutoff
    d = F.parse_definition("LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 "
                           "-algorithm NonbondedCutoff -switchon 7 -cutoff 10 -cutoff 8 -cutoff 11")
    assert d["terms"][0][2:4] == (7.0, 10.0)
    assert d["terms"][1][3] == 8.0
    assert d["algo_cutoff"] == 11.0


def test_parse_reuses_a_keyword_after_wrapping_around():
    # the reference scans once more from the start when a keyword is not
    # found after the previous match (ForceFactoryDetails.cpp:209-221)
    d = F.parse_definition("LennardJones -switchingFunction C2 -algorithm NonbondedCutoff -switchon 8 -cutoff 9")
    assert d["algo_cutoff"] == 9.0


@pytest.mark.parametrize("bad", [
    "LennardJones -switchingFunction C2 -algorithm NonbondedCutoff -switchon 8",
    "Bogus -algorithm NonbondedCutoff",
    "Coulomb -algorithm PMEwald -interpolation Hermite -gridsize 8 8 8 -cutoff 9",
    "LennardJones -algorithm Nowhere",
])
def test_parse_rejects_incomplete_definitions(bad):
    with pytest.raises(ValueError):
        F.parse_definition(bad)


@pytest.mark.parametrize("bad", [
    # ProtoMol registers PMEwald with the Cutoff switch only
    # (registerForceExemplarsFastElectrostatic.cpp:50-55): a Shift or C2 line
    # finds no exemplar
    "Coulomb -algorithm PMEwald -real -reciprocal -correction -switchingFunction Shift "
    "-interpolation BSpline -gridsize 8 8 8 -cutoff 9",
    "Coulomb -algorithm PMEwald -real -reciprocal -correction -switchingFunction C2 "
    "-interpolation BSpline -gridsize 8 8 8 -cutoff 9",
    # no term at all, and -real -reciprocal without -correction: not registered
    "Coulomb -algorithm PMEwald -interpolation BSpline -gridsize 8 8 8 -cutoff 9",
    "Coulomb -algorithm PMEwald -real -reciprocal -interpolation BSpline -gridsize 8 8 8 -cutoff 9",
])
def test_parse_rejects_unregistered_pme_variants(bad):
    with pytest.raises(ValueError, match="Could not find a complete match"):
        F.parse_definition(bad)


@pytest.mark.parametrize("flags", ["-real -reciprocal -correction", "-real", "-real -correction",
                                   "-reciprocal", "-reciprocal -correction", "-correction"])
def test_parse_accepts_every_registered_pme_variant(flags):
    d = F.parse_definition(f"Coulomb -algorithm PMEwald {flags} -interpolation BSpline -gridsize 8 8 8 -cutoff 9")
    assert (d["real"], d["reciprocal"], d["correction"]) == tuple(int(f"-{t}" in flags.split())
                                                                 for t in ("real", "reciprocal", "correction"))
    # the Cutoff switch may be written out
    F.parse_definition(f"Coulomb -algorithm PMEwald {flags} -switchingFunction Cutoff -interpolation BSpline "
                       "-gridsize 8 8 8 -cutoff 9")
