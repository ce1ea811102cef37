"""The launch-shape autotuner (pmgpu_autotune, pmgpu_batch_autotune) and the
tunings it chooses between: every candidate value gives the same forces,
energies and virial up to the grouping of a chunk's partial sums, and a tuned
system still matches the oracle."""
import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import _lib
from protomol_b200 import forces as F
from protomol_b200 import systems, workloads

pytestmark = pytest.mark.gpu

CANDIDATES = [dict(chunk_entries=8), dict(chunk_entries=32), dict(pair_blocks_per_sm=2),
              dict(pair_blocks_per_sm=3), dict(fft_lines=4), dict(fft_lines=8), dict(pme_concurrent=0)]


def small_pme_box():
    # 3,060 atoms, cutoff 9 + PME 32^3 (the cutoff + PME path of every tunable)
    s = systems.chain_in_water(n_chain=60, n_water=1000, length=32.0, seed=21)
    defs = [workloads.lj_ewald_split(7, 9, 0.35), workloads.pme_reciprocal((32, 32, 32), 9, 0.35)]
    return s, defs


def run(topo, fs, s):
    out = np.zeros((s.n_atoms, 3))
    e = F.ScalarStructure()
    F.evaluate_group(topo, fs, s.positions, out, e)
    return out, e


def test_set_and_get_tuning_round_trip_and_reject_out_of_range():
    s, defs = small_pme_box()
    topo = F.Topology(s)
    t = topo.tuning
    assert (t["chunk_entries"], t["pair_blocks_per_sm"], t["fft_lines"], t["pme_concurrent"],
            t["fp64_pairs"]) == (16, 0, 16, 1, 0)
    topo.set_tuning(chunk_entries=32, fft_lines=4)
    assert topo.tuning["chunk_entries"] == 32 and topo.tuning["fft_lines"] == 4
    for bad in (dict(chunk_entries=2), dict(chunk_entries=128), dict(pair_blocks_per_sm=-1),
                dict(fft_lines=0), dict(fft_lines=17), dict(pme_concurrent=2), dict(fp64_pairs=2)):
        with pytest.raises(_lib.PmgpuError):
            topo.set_tuning(**bad)
    assert topo.tuning["chunk_entries"] == 32                  # unchanged by a rejected call
    topo.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_every_candidate_tuning_gives_the_same_result(precision):
    s, defs = small_pme_box()
    topo = F.Topology(s)
    fs = [F.ForceFactory.make(topo, d, precision) for d in defs]
    f0, e0 = run(topo, fs, s)
    rms = np.sqrt((f0 ** 2).sum(1).mean())
    scale = abs(e0.lennard_jones) + abs(e0.coulomb)
    base = topo.tuning
    # Mixed: a chunk's i-forces are FP32 register sums before their fixed-point
    # rounding, so another chunking regroups FP32 additions (~1e-7 relative
    # RMS; the force bound against FP64 is 1e-5), and the chunk-lane energy
    # partials are rounded to 2^-32 in other groups (~1e-12 relative).  FP64:
    # only the fixed-point grouping.
    ftol, etol, vtol = (1e-6, 1e-10, 1e-6) if precision == "mixed" else (1e-9, 1e-12, 1e-11)
    bad = []
    for cand in CANDIDATES:
        topo.set_tuning(**{**{k: base[k] for k in ("chunk_entries", "pair_blocks_per_sm", "fft_lines",
                                                    "pme_concurrent")}, **cand})
        f, e = run(topo, fs, s)
        errs = {"force": np.sqrt(((f - f0) ** 2).sum() / (f0 ** 2).sum()) if precision == "mixed"
                else np.abs(f - f0).max() / rms,
                "lj": abs(e.lennard_jones - e0.lennard_jones) / scale,
                "coulomb": abs(e.coulomb - e0.coulomb) / scale,
                "virial": np.abs(e.virial_tensor - e0.virial_tensor).max() / np.abs(e0.virial_tensor).max()}
        tol = {"force": ftol, "lj": etol, "coulomb": etol, "virial": vtol}
        bad += [(cand, k, v) for k, v in errs.items() if not v <= tol[k]]
    assert not bad, bad
    topo.close()


@pytest.mark.parametrize("which", ["water216", "small_pme"])
def test_fp64_pairs_gives_the_fp64_kernels_results(which):
    """fp64_pairs = 1 runs a mixed cutoff force on the FP64 pair kernels (the
    shorter launch chain the autotuner may pick for a few hundred atoms):
    its forces, energies and virial are the FP64 force's, bit for bit, and
    the layout reads 'fp64'; back at 0 the mixed kernels run again."""
    if which == "water216":
        w = workloads.water216()
        s, defs = w.system, w.forces
    else:
        s, defs = small_pme_box()
    outs = {}
    for prec in ("fp64", "mixed"):
        topo = F.Topology(s)
        fs = [F.ForceFactory.make(topo, d, prec) for d in defs]
        if prec == "mixed":
            fm, em = run(topo, fs, s)
            assert topo.pair_layout() in ("cells", "columns")
            topo.set_tuning(fp64_pairs=1)
        outs[prec] = run(topo, fs, s)
        if prec == "mixed":
            assert topo.pair_layout() == "fp64"
            topo.set_tuning(fp64_pairs=0)
            f2, e2 = run(topo, fs, s)
            assert topo.pair_layout() in ("cells", "columns")
            assert np.array_equal(f2, fm) and e2.lennard_jones == em.lennard_jones
        topo.close()
    (fd, ed), (fx, ex) = outs["fp64"], outs["mixed"]
    if which == "water216":
        # cutoff forces alone: the same kernels on the same inputs
        assert np.array_equal(fd, fx)
        assert ed.lennard_jones == ex.lennard_jones and ed.coulomb == ex.coulomb
        assert np.array_equal(ed.virial_tensor, ex.virial_tensor)
    else:
        # the PME force stays mixed: the pair part is the FP64 one, the sum
        # within the mixed bounds of the FP64 result
        assert np.sqrt(((fx - fd) ** 2).sum() / (fd ** 2).sum()) <= 1e-5
        assert abs(ed.lennard_jones - ex.lennard_jones) <= 1e-12 * abs(ed.lennard_jones)


def test_autotuned_system_matches_the_oracle():
    s, defs = small_pme_box()
    topo = F.Topology(s)
    fs = [F.ForceFactory.make(topo, d, "mixed") for d in defs]
    best = topo.autotune(fs, s.positions, evals=3)
    assert 4 <= best["chunk_entries"] <= 64 and 1 <= best["fft_lines"] <= 16
    assert best["pme_concurrent"] in (0, 1) and best["ms_per_eval"] > 0
    assert topo.tuning == best                                 # kept for the later evaluations
    ref = oracle.evaluate(s, [F.parse_definition(d) for d in defs])
    f, e = run(topo, fs, s)
    assert np.sqrt(((f - ref["forces"]) ** 2).sum() / (ref["forces"] ** 2).sum()) <= 1e-5
    scale = abs(ref["lennard_jones"]) + abs(ref["coulomb"])
    assert abs(e.lennard_jones + e.coulomb - ref["lennard_jones"] - ref["coulomb"]) <= 2e-6 * scale
    topo.close()


def test_batch_autotune_then_members_equal_their_own_evaluation():
    from protomol_b200.batch import Batch
    ws = [workloads.water_box_workload(n, 70 + k) for k, n in enumerate([150, 600, 1400])]
    batch = Batch(0)
    alone = []
    for w in ws:
        topo = F.Topology(w.system)
        fs = [F.ForceFactory.make(topo, d, "mixed") for d in w.forces]
        batch.add(topo, fs, w.system.positions)
        alone.append((topo, fs, w.system))
    best = batch.autotune(evals=2)
    assert best["ms_per_eval"] > 0
    batch.evaluate()
    for (fb, eb), (topo, fs, s) in zip(batch.results(), alone):
        assert topo.tuning == best
        fa, ea = run(topo, fs, s)                              # alone, same tuning: bitwise
        assert np.array_equal(fb, fa)
        assert eb.lennard_jones == ea.lennard_jones and eb.coulomb == ea.coulomb
    batch.close()
