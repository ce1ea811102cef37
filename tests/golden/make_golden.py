"""Generates the golden fixtures in this directory from the REFERENCE itself.

    python tests/golden/make_golden.py [case ...]

Needs oracle/_ref/pmref (built from the ProtoMol sources by
``make -C oracle/ref``), i.e. it runs where the reference sources exist.  For
each case it runs the reference's own NonbondedCutoffSystemForce /
NonbondedPMEwaldSystemForce on a seeded system from
``protomol_b200.systems`` and stores the energies, the virial, the cell
assignment and the forces (all atoms for the two main cases, 64 sampled
atoms otherwise).  The systems themselves are regenerated from their seeds;
``pos_sha`` pins that the generator still produces the same coordinates.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from protomol_b200 import forces as F  # noqa: E402
from protomol_b200 import systems, workloads  # noqa: E402


def cases():
    """name -> (system factory, [force definitions], store all forces)"""
    small = lambda: systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)

    def small_csf():             # coulombScalingFactor 1: the 1-4 pairs unscaled
        s = small()
        s.csf = 1.0
        return s

    wb = lambda: systems.water_box(100, seed=7)
    alpha_s = 0.35
    return {
        "water216_c2": (systems.water_box_216, workloads.water216().forces, True),
        "small_split_pme": (small, [workloads.lj_ewald_split(7, 9, alpha_s),
                                    workloads.pme_reciprocal((24, 24, 24), 9, alpha_s)], True),
        "small_c1lj_ewald": (small, ["LennardJones CoulombEwaldReal -switchingFunction C1 -switchingFunction Cutoff "
                                     "-algorithm NonbondedCutoff -cutoff 9 -alpha 0.35 -cutoff 9 -cutoff 9"], False),
        "small_c2lj_c1coul": (small, ["LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 "
                                      "-algorithm NonbondedCutoff -switchon 7 -cutoff 10 -cutoff 8 -cutoff 10"], False),
        "small_c2lj_shiftcoul": (small, ["LennardJones Coulomb -switchingFunction C2 -switchingFunction Shift "
                                         "-algorithm NonbondedCutoff -switchon 7 -cutoff 9 -cutoff 10 -cutoff 10"], False),
        "small_cutlj_cutewald": (small, ["LennardJones CoulombEwaldReal -switchingFunction Cutoff -switchingFunction "
                                         "Cutoff -algorithm NonbondedCutoff -cutoff 8 -alpha 0.35 -cutoff 9 -cutoff 9"],
                                 False),
        "small_c2_fused": (small, ["LennardJones Coulomb -switchingFunction C2 -switchingFunction C2 -algorithm "
                                   "NonbondedCutoff -switchon 8 -cutoff 9 -switchon 6 -cutoff 9 -cutoff 9"], False),
        "small_shift_lj": (small, ["LennardJones -switchingFunction Shift -algorithm NonbondedCutoff -cutoff 9 -cutoff 9"],
                           False),
        "small_cutoff_coulomb": (small, ["Coulomb -switchingFunction Cutoff -algorithm NonbondedCutoff -cutoff 9 "
                                         "-cutoff 9"], False),
        "small_pme_default_alpha": (small, ["Coulomb -algorithm PMEwald -reciprocal -correction -interpolation BSpline "
                                            "-gridsize 25 27 30 -cutoff 9"], False),
        # look-up-table potentials (registerForceExemplarsCutoff.cpp:47-48,58,69,86,101,132-134)
        "small_table_lj_c2": (small, ["LennardJonesTable -switchingFunction C2 -algorithm NonbondedCutoff "
                                      "-switchon 7 -cutoff 9 -cutoff 9"], False),
        "small_table_coulomb_shift": (small, ["CoulombTable -switchingFunction Shift -algorithm NonbondedCutoff "
                                              "-cutoff 9 -cutoff 9"], False),
        "small_csf1_table_coulomb_cutoff": (small_csf, ["CoulombTable -switchingFunction Cutoff -algorithm "
                                                       "NonbondedCutoff -cutoff 9 -cutoff 9"], False),
        "small_table_ewald": (small, ["CoulombEwaldRealTable -algorithm NonbondedCutoff -cutoff 9 -alpha 0.35 "
                                      "-cutoff 9"], False),
        "small_table_c2lj_ewald": (small, ["LennardJones CoulombEwaldRealTable -switchingFunction C2 -algorithm "
                                           "NonbondedCutoff -switchon 7 -cutoff 10 -cutoff 8.5 -alpha 0.35 "
                                           "-cutoff 10"], False),
        "small_csf1_table_c1lj_ewald": (small_csf, ["LennardJones CoulombEwaldRealTable -switchingFunction C1 "
                                                   "-algorithm NonbondedCutoff -cutoff 9 -cutoff 9 -alpha 0.35 "
                                                   "-cutoff 9"], False),
        "small_table_ljt_ewald": (small, ["LennardJonesTable CoulombEwaldRealTable -switchingFunction C2 "
                                          "-algorithm NonbondedCutoff -switchon 8 -cutoff 9 -cutoff 10 -alpha 0.3 "
                                          "-cutoff 10"], False),
        "small_table_ljt_coult": (small, ["LennardJonesTable CoulombTable -switchingFunction C2 -switchingFunction "
                                          "Shift -algorithm NonbondedCutoff -switchon 1 -cutoff 9 -cutoff 9.5 "
                                          "-cutoff 9.5"], False),
        "smallbox_wrap": (wb, workloads.water_box_workload(100, 7).forces, True),
    }


def pos_sha(s) -> str:
    return hashlib.sha256(np.ascontiguousarray(s.positions).tobytes()).hexdigest()[:16]


def main(only=()):
    if not oracle.reference_available():
        raise SystemExit("oracle/_ref/pmref missing: make -C oracle/ref")
    for name, (factory, defs, full) in cases().items():
        if only and name not in only:
            continue
        s = factory()
        specs = [F.parse_definition(d) for d in defs]
        r = oracle.run_reference(s, specs)
        rng = np.random.default_rng(0)
        idx = np.arange(s.n_atoms) if full else np.sort(rng.choice(s.n_atoms, 64, replace=False))
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            definitions=np.array(defs), pos_sha=np.array(pos_sha(s)), n_atoms=s.n_atoms,
            lennard_jones=r["lennard_jones"], coulomb=r["coulomb"], virial=r["virial"],
            force_index=idx, forces=r["forces"][idx], cells=r["cells"], dims=np.array(r["dims"]),
            force_rms=np.sqrt((r["forces"] ** 2).sum(1).mean()),
        )
        print(name, s.n_atoms, r["lennard_jones"], r["coulomb"])


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))     # names of the cases to regenerate (default: all)
