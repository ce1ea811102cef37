"""The named workloads: a system plus the force definitions ProtoMol's
``.conf`` would give for it (keyword strings of ``ForceFactory``)."""
from __future__ import annotations

from dataclasses import dataclass, field

from . import systems


@dataclass
class Workload:
    name: str
    system: object
    forces: list = field(default_factory=list)   # force definition strings, evaluated in order


def lj_c2_coulomb_c2(on: float, rc: float):
    return [
        f"LennardJones -switchingFunction C2 -algorithm NonbondedCutoff -switchon {on} -cutoff {rc} -cutoff {rc}",
        f"Coulomb -switchingFunction C2 -algorithm NonbondedCutoff -switchon {on} -cutoff {rc} -cutoff {rc}",
    ]


def lj_ewald_split(on: float, rc: float, alpha: float):
    return (f"LennardJones CoulombEwaldReal -switchingFunction C2 -switchingFunction Cutoff "
            f"-algorithm NonbondedCutoff -switchon {on} -cutoff {rc} -alpha {alpha} -cutoff {rc} -cutoff {rc}")


def pme_reciprocal(grid, rc: float, alpha: float, order: int = 4):
    gx, gy, gz = grid
    return (f"Coulomb -algorithm PMEwald -reciprocal -correction -interpolation BSpline "
            f"-gridsize {gx} {gy} {gz} -cutoff {rc} -order {order} -alpha {alpha}")


def water216() -> Workload:
    """216 TIP3P waters, LJ + Coulomb, both C2 8 -> 9 A (two forces)."""
    return Workload("water216_cutoff_c2", systems.water_box_216(), lj_c2_coulomb_c2(8, 9))


def chain14281() -> Workload:
    """14,281-atom chain in water: LJ C2 10 -> 12 + Ewald real (Cutoff 12,
    alpha 0.32) in one cutoff force, plus PME 64^3 order 4 reciprocal +
    correction."""
    return Workload("chain14281_cutoff_pme", systems.chain_in_water_14281(),
                    [lj_ewald_split(10, 12, 0.32), pme_reciprocal((64, 64, 64), 12, 0.32)])


def water1m() -> Workload:
    """1,000,000 atoms: cutoff 12 (C2 10 -> 12) + PME 216^3, alpha 0.32."""
    return Workload("water1M_cutoff_pme", systems.water_box_1m(),
                    [lj_ewald_split(10, 12, 0.32), pme_reciprocal((216, 216, 216), 12, 0.32)])


def lj_fluid216() -> Workload:
    """216 LJ oxygens (the 648-atom water box without its hydrogens), LJ C2
    8 -> 9 A: the Leapfrog runs of the plain-cutoff configuration."""
    return Workload("oxygen216_lj_c2", systems.oxygen_fluid_216(),
                    ["LennardJones -switchingFunction C2 -algorithm NonbondedCutoff -switchon 8 -cutoff 9 -cutoff 9"])


def water_box_workload(n_water: int, seed: int) -> Workload:
    """One of the batched boxes: cutoff 9 (C2 8 -> 9), alpha from the default
    accuracy 1e-6, PME grid ~1 A rounded to 2^a 3^b 5^c."""
    s = systems.water_box(n_water, seed)
    alpha = systems.ewald_alpha(9.0)
    k = systems.smooth_grid_size(float(s.box[0, 0]))
    return Workload(f"water{n_water}", s, [lj_ewald_split(8, 9, alpha), pme_reciprocal((k, k, k), 9, alpha)])


def batched96(count: int = 96, seed: int = 4):
    import numpy as np
    rng = np.random.default_rng(seed)
    sizes = rng.integers(100, 3001, count)
    return [water_box_workload(int(n), 1000 + k) for k, n in enumerate(sizes)]
