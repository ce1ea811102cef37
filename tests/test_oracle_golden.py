"""The CPU restatement (oracle/pmoracle.c) against golden vectors produced by
the reference itself (tests/golden/make_golden.py runs ProtoMol's own force
classes built from its sources).  CPU only."""
import hashlib
import os

import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import forces as F
from protomol_b200 import systems

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _case_system(name):
    if name == "water216_c2":
        return systems.water_box_216()
    if name == "smallbox_wrap":
        return systems.water_box(100, seed=7)
    s = systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)
    if "_csf1" in name:
        s.csf = 1.0
    return s


CASES = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    s = _case_system(name)
    assert hashlib.sha256(np.ascontiguousarray(s.positions).tobytes()).hexdigest()[:16] == str(g["pos_sha"])
    specs = [F.parse_definition(str(d)) for d in g["definitions"]]
    r = oracle.evaluate(s, specs)
    # energies and virial: same operation order as the reference; only the
    # FFT (ZFFT vs the restatement's mixed-radix DFT) rounds differently
    scale = abs(float(g["lennard_jones"])) + abs(float(g["coulomb"])) + 1.0
    assert abs(r["lennard_jones"] - float(g["lennard_jones"])) <= 1e-11 * scale
    assert abs(r["coulomb"] - float(g["coulomb"])) <= 1e-11 * scale
    vs = np.abs(g["virial"]).max() + 1.0
    assert np.abs(r["virial"] - g["virial"]).max() <= 1e-11 * vs
    f = r["forces"][g["force_index"]]
    assert np.abs(f - g["forces"]).max() <= 1e-11 * max(float(g["force_rms"]), 1.0)
    cells, dims, oog = oracle.cell_assign(s)
    assert dims == tuple(int(x) for x in g["dims"])
    assert np.array_equal(cells, g["cells"])
    assert oog == 0


def test_cutoff_cases_are_bit_exact_with_reference_golden():
    """Without an FFT in the path the restatement reproduces the reference
    bit for bit."""
    for name in ["water216_c2", "small_c2lj_c1coul", "small_c2_fused", "small_cutoff_coulomb"] + \
            [c for c in CASES if "table" in c]:
        g = np.load(os.path.join(GOLDEN, name + ".npz"))
        s = _case_system(name)
        r = oracle.evaluate(s, [F.parse_definition(str(d)) for d in g["definitions"]])
        assert r["lennard_jones"] == float(g["lennard_jones"])
        assert r["coulomb"] == float(g["coulomb"])
        assert np.array_equal(r["virial"], g["virial"])
        assert np.array_equal(r["forces"][g["force_index"]], g["forces"])


def test_poly5_is_the_abramowitz_stegun_polynomial():
    # erfc(x) ~ poly5(x) exp(-x^2), |error| <= 1.5e-7 (A&S 7.1.26)
    import math
    for x in np.linspace(0.0, 4.0, 81):
        assert abs(oracle.poly5(x) * math.exp(-x * x) - math.erfc(x)) <= 1.5e-7


def test_fft_restatement_against_numpy():
    rng = np.random.default_rng(0)
    a = rng.normal(size=(6, 10, 15)) + 1j * rng.normal(size=(6, 10, 15))
    assert np.allclose(oracle.fft3d(a, -1), np.fft.fftn(a), atol=1e-10)
    assert np.allclose(oracle.fft3d(a, +1), np.fft.ifftn(a) * a.size, atol=1e-10)


def test_pair_set_of_restatement_is_unordered_unique():
    s = systems.water_box_216()
    r = oracle.evaluate(s, [F.parse_definition(
        "LennardJones -switchingFunction C2 -algorithm NonbondedCutoff -switchon 8 -cutoff 9 -cutoff 9")],
        want_pairs=True)
    p = r["pairs"]
    assert (p[:, 0] < p[:, 1]).all()
    keys = p[:, 0].astype(np.int64) * s.n_atoms + p[:, 1]
    assert len(np.unique(keys)) == len(keys) == r["n_pairs"]
    # brute force: minimal-image pairs within 9 A that are not excluded
    d = s.positions[:, None, :] - s.positions[None, :, :]
    L = s.box_lengths
    d -= L * np.rint(d / L)
    r2 = (d * d).sum(-1)
    iu = np.triu_indices(s.n_atoms, 1)
    within = r2[iu] <= 81.0
    same = s.molecule[iu[0]] == s.molecule[iu[1]]
    assert within.sum() - (within & same).sum() == len(keys)
