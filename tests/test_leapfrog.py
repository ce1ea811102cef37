"""The Leapfrog integrator on device-resident state (pmgpu_leapfrog_run)
against the oracle's restatement of LeapfrogIntegrator::run, 1 fs steps from
seeded 300 K Maxwell-Boltzmann velocities:

* ten steps of the 648-atom water box of the plain-cutoff configuration
  (LJ + Coulomb, C2 8 -> 9 A, intra-water pairs excluded);
* one force evaluation plus 1,000 steps of the same box's 216 oxygens as a
  Lennard-Jones fluid;
* the configuration as stated: the 216 waters held rigid by ProtoMol's
  SHAKE (post-drift) and RATTLE (post-step) modifiers, one force evaluation
  plus 1,000 steps.  The oracle's constrained Leapfrog is pinned bit for
  bit to ProtoMol's own LeapfrogIntegrator with ModifierShake and
  ModifierRattle (protomol_b200/adapter's gpu_leapfrog_driver on the
  reference forces)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import forces as F
from protomol_b200 import integrate, workloads

from protomol_b200 import systems

DT = 1.0                     # fs
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LEAPFROG = os.path.join(ROOT, "protomol_b200", "adapter", "_build", "gpu_leapfrog_driver")
# protomol.cpp:137-141 defaults: epsilon 1e-5, 30 sweeps
RIGID = {"shake": (1e-5, 30), "rattle": (1e-5, 30)}


def rigid_constraints(system, shake=(1e-5, 30), rattle=(1e-5, 30)):
    atoms, rest = systems.rattle_shake_constraints(system)
    return {"atoms": atoms, "rest": rest, "mass": system.mass, "shake": shake, "rattle": rattle}


def reference_constrained_leapfrog(system, defs, v, steps, shake, rattle):
    """ProtoMol's LeapfrogIntegrator with its SHAKE / RATTLE modifiers on the
    reference forces (gpu_leapfrog_driver, cpu mode)."""
    with tempfile.TemporaryDirectory() as td:
        sp, dp, op, cp = (os.path.join(td, f) for f in ("s.bin", "d.bin", "o.bin", "c.txt"))
        system.save(sp)
        np.concatenate([system.mass, v.ravel()]).astype(np.float64).tofile(dp)
        _, rest = systems.rattle_shake_constraints(system)
        se, si = shake or (0.0, 0)
        re_, ri = rattle or (0.0, 0)
        with open(cp, "w") as fh:
            fh.write(f"{len(system.bonds)} {len(system.angles)} {float(se)!r} {si} {float(re_)!r} {ri}\n")
            for (b1, b2), r in zip(system.bonds, rest):
                fh.write(f"{b1} {b2} {float(r)!r}\n")
            for a1, a2, a3 in system.angles:
                fh.write(f"{a1} {a2} {a3} {systems._HOH!r}\n")
        p = subprocess.run([LEAPFROG, sp, dp, op, str(steps), repr(DT), "cpu", *defs], capture_output=True, text=True,
                           timeout=600, env=dict(os.environ, LF_CONSTRAINTS=cp))
        assert p.returncode == 0, p.stderr
        raw = np.fromfile(op)
    n = system.n_atoms
    return raw[2:2 + 3 * n].reshape(n, 3), raw[2 + 3 * n:].reshape(n, 3), raw[0]


@pytest.mark.skipif(not os.path.exists(LEAPFROG), reason="the ProtoMol-side driver is not built here")
@pytest.mark.parametrize("shake,rattle", [((1e-5, 30), None), ((1e-5, 30), (1e-5, 30)), ((1e-8, 100), (1e-8, 100))])
def test_oracle_constrained_leapfrog_is_the_reference(shake, rattle):
    w, v = water648()
    specs = [F.parse_definition(d) for d in w.forces]
    x, v1, f, r = oracle.leapfrog(w.system, specs, v, DT, 20, constraints=rigid_constraints(w.system, shake, rattle))
    xr, vr, epot = reference_constrained_leapfrog(w.system, w.forces, v, 20, shake, rattle)
    assert np.array_equal(x, xr) and np.array_equal(v1, vr)
    assert epot == r["lennard_jones"] + r["coulomb"]


def water648():
    w = workloads.water216()
    v = integrate.maxwell_boltzmann(w.system.mass, 300.0, seed=648)
    return w, v


def oxygen_fluid():
    w = workloads.lj_fluid216()
    return w, integrate.maxwell_boltzmann(w.system.mass, 300.0, seed=216)


def test_maxwell_boltzmann_velocities_have_the_temperature():
    w, v = water648()
    n = w.system.n_atoms
    # 3N - 3 degrees of freedom after removing the net momentum
    t = 2.0 * integrate.kinetic_energy(w.system.mass, v) / ((3 * n - 3) * integrate.BOLTZMANN)
    assert abs(t - 300.0) < 300.0 * 4.0 / np.sqrt(3 * n)       # within ~4 sigma of the sample
    assert np.abs((w.system.mass[:, None] * v).sum(0)).max() < 1e-9


def test_oracle_leapfrog_conserves_energy():
    w, v = oxygen_fluid()
    specs = [F.parse_definition(d) for d in w.forces]
    r0 = oracle.evaluate(w.system, specs)
    e0 = r0["lennard_jones"] + r0["coulomb"] + integrate.kinetic_energy(w.system.mass, v)
    x, v1, f, r = oracle.leapfrog(w.system, specs, v, DT, 40, forces=r0["forces"])
    e1 = r["lennard_jones"] + r["coulomb"] + integrate.kinetic_energy(w.system.mass, v1)
    ke = integrate.kinetic_energy(w.system.mass, v)
    assert abs(e1 - e0) < 0.01 * ke


def _gpu_run(w, v, precision, chunks):
    topo = F.Topology(w.system)
    fs = [F.ForceFactory.make(topo, d, precision) for d in w.forces]
    lf = integrate.Leapfrog(topo, fs, w.system.positions, v, w.system.mass, DT).initialize()
    out = []
    for n in chunks:
        lf.run(n)
        out.append(lf.state())
    return topo, out


@pytest.mark.gpu
def test_ten_steps_match_the_oracle():
    w, v = water648()
    specs = [F.parse_definition(d) for d in w.forces]
    x, v1, f, r = oracle.leapfrog(w.system, specs, v, DT, 10)
    _, [(xg, vg, fg, eg)] = _gpu_run(w, v, "fp64", [10])
    print(f"\n10 steps: |dx| {np.abs(xg - x).max():.2e} A  |dv| {np.abs(vg - v1).max():.2e}  "
          f"|dF| {np.abs(fg - f).max():.2e}")
    # the FP64 forces agree with the oracle to ~1e-12; ten steps keep that
    assert np.abs(xg - x).max() <= 1e-10
    assert np.abs(vg - v1).max() <= 1e-10 * np.abs(v1).max()
    assert np.abs(fg - f).max() <= 1e-8 * np.sqrt((f ** 2).sum(1).mean())
    assert abs(eg.lennard_jones + eg.coulomb - r["lennard_jones"] - r["coulomb"]) <= 1e-9 * (
        abs(r["lennard_jones"]) + abs(r["coulomb"]))


@pytest.mark.gpu
def test_one_evaluation_plus_a_thousand_steps():
    """One evaluation plus 1,000 steps, FP64 on the GPU against the oracle:
    the trajectories separate only by the amplified rounding of the forces (a
    fluid's trajectories diverge exponentially), and both conserve the total
    energy alike."""
    w, v = oxygen_fluid()
    specs = [F.parse_definition(d) for d in w.forces]
    r0 = oracle.evaluate(w.system, specs)
    x, v1, f, r = oracle.leapfrog(w.system, specs, v, DT, 1000, forces=r0["forces"])
    _, [(xg, vg, fg, eg)] = _gpu_run(w, v, "fp64", [1000])
    ke0 = integrate.kinetic_energy(w.system.mass, v)
    e0 = r0["lennard_jones"] + r0["coulomb"] + ke0
    e_ref = r["lennard_jones"] + r["coulomb"] + integrate.kinetic_energy(w.system.mass, v1)
    e_gpu = eg.lennard_jones + eg.coulomb + integrate.kinetic_energy(w.system.mass, vg)
    print(f"\n1000 steps: |dx| {np.abs(xg - x).max():.2e} A  energy drift oracle {e_ref - e0:+.4f} "
          f"gpu {e_gpu - e0:+.4f} kcal/mol (KE {ke0:.1f})")
    # measured: 1.6e-11 A apart after 1,000 steps, the same energy drift
    assert np.abs(xg - x).max() <= 1e-8
    assert abs(e_gpu - e_ref) <= 1e-6 * ke0
    assert abs(e_gpu - e0) <= 0.01 * ke0


@pytest.mark.gpu
def test_mixed_precision_trajectory_conserves_energy_like_fp64():
    w, v = oxygen_fluid()
    ke0 = integrate.kinetic_energy(w.system.mass, v)
    drifts = {}
    for precision in ("fp64", "mixed"):
        topo, states = _gpu_run(w, v, precision, [100] * 10)
        e = [s[3].lennard_jones + s[3].coulomb + integrate.kinetic_energy(w.system.mass, s[1]) for s in states]
        drifts[precision] = np.ptp(e)
    print(f"\ntotal energy range over 1000 steps: fp64 {drifts['fp64']:.4f}  mixed {drifts['mixed']:.4f} "
          f"kcal/mol (KE {ke0:.1f})")
    assert drifts["mixed"] <= 2.0 * drifts["fp64"] + 1e-3 * ke0


# ---------------------------------------------------------------- Impulse (MTS)
FAST = "LennardJones -switchingFunction C2 -algorithm NonbondedCutoff -switchon 8 -cutoff 9 -cutoff 9"
SLOW = ("Coulomb -algorithm PMEwald -real -reciprocal -correction -interpolation BSpline -gridsize 20 20 20 "
        "-cutoff 8.5 -alpha 0.35")


@pytest.mark.gpu
def test_impulse_matches_the_oracle():
    """ImpulseIntegrator over Leapfrog, PME as the slow force: 10 outer steps
    of 4 x 0.5 fs on the 216-particle ionic fluid, FP64 on the GPU against the
    oracle's restatement."""
    from protomol_b200 import systems
    s = systems.ionic_fluid_216()
    v = integrate.maxwell_boltzmann(s.mass, 300.0, seed=21)
    slow, fast = [F.parse_definition(SLOW)], [F.parse_definition(FAST)]
    x, v1, fs, ff, epot = oracle.impulse(s, slow, fast, v, 0.5, 4, 10)
    topo = F.Topology(s)
    imp = integrate.Impulse(topo, [F.ForceFactory.make(topo, SLOW, "fp64")], [F.ForceFactory.make(topo, FAST, "fp64")],
                            s.positions, v, s.mass, 0.5, 4).initialize().run(10)
    xg, vg, fsg, ffg, eg = imp.state()
    print(f"\nimpulse 10 x 4 steps: |dx| {np.abs(xg - x).max():.2e} A  |dv| {np.abs(vg - v1).max():.2e}  "
          f"dE {eg - epot:+.2e}")
    assert np.abs(xg - x).max() <= 1e-10
    assert np.abs(vg - v1).max() <= 1e-10 * np.abs(v1).max()
    assert np.abs(fsg - fs).max() <= 1e-8 * np.sqrt((fs ** 2).sum(1).mean())
    assert abs(eg - epot) <= 1e-9 * abs(epot)


@pytest.mark.gpu
def test_impulse_with_cyclelength_one_is_leapfrog_with_all_forces():
    """One inner step per outer step: the same trajectory as a Leapfrog on
    the sum of the two groups, up to the order of the kicks' additions."""
    from protomol_b200 import systems
    s = systems.ionic_fluid_216()
    v = integrate.maxwell_boltzmann(s.mass, 300.0, seed=22)
    topo = F.Topology(s)
    slow, fast = F.ForceFactory.make(topo, SLOW, "fp64"), F.ForceFactory.make(topo, FAST, "fp64")
    imp = integrate.Impulse(topo, [slow], [fast], s.positions, v, s.mass, 1.0, 1).initialize().run(20)
    xi = imp.state()[0]
    lf = integrate.Leapfrog(topo, [slow, fast], s.positions, v, s.mass, 1.0).initialize().run(20)
    xl = lf.state()[0]
    assert np.abs(xi - xl).max() <= 1e-9


# ---------------------------------------------------------------- rigid water
def _gpu_rigid(w, v, precision, steps, virial=False):
    topo = F.Topology(w.system)
    fs = [F.ForceFactory.make(topo, d, precision) for d in w.forces]
    lf = integrate.Leapfrog(topo, fs, w.system.positions, v, w.system.mass, DT, virial=virial,
                            constraints=rigid_constraints(w.system)).initialize()
    lf.run(steps)
    return lf.state(), lf.constraint_limit_hits()


@pytest.mark.gpu
def test_rigid_water_ten_steps_match_the_oracle():
    """SHAKE and RATTLE on the GPU against the oracle (itself the reference's
    integrator bit for bit), FP64 forces; with the virial, RATTLE's final
    term included."""
    w, v = water648()
    specs = [F.parse_definition(d) for d in w.forces]
    x, v1, f, r = oracle.leapfrog(w.system, specs, v, DT, 10, constraints=rigid_constraints(w.system))
    (xg, vg, fg, eg), hits = _gpu_rigid(w, v, "fp64", 10, virial=True)
    print(f"\nrigid water, 10 steps: |dx| {np.abs(xg - x).max():.2e} A  |dv| {np.abs(vg - v1).max():.2e}")
    assert hits == 0
    assert np.abs(xg - x).max() <= 1e-10
    assert np.abs(vg - v1).max() <= 1e-10 * np.abs(v1).max()
    assert np.abs(eg.virial_tensor - r["virial"]).max() <= 1e-8 * np.abs(r["virial"]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rigid_water_one_evaluation_plus_a_thousand_steps(precision):
    """The plain-cutoff configuration as stated: 216 rigid TIP3P waters, one
    evaluation plus 1,000 steps of 1 fs.  The lattice's random orientations
    heat the box (the kinetic energy grows from ~530 to ~7,800 kcal/mol),
    after which the total energy creeps up by the 1 fs step's error at that
    temperature: from step 100 to step 1,000 the oracle's runs gain +38 to
    +81 kcal/mol (0.5-1% of the kinetic energy) depending on the realization
    (velocities scaled by 1 + k 1e-12 separate after ~300 steps).  Over four
    such realizations the GPU's mean gain stays below 2% of the kinetic
    energy, the bonds stay at their rest lengths within SHAKE's tolerance,
    and the unscaled FP64 run follows the oracle's over the first 100 steps."""
    w, v = water648()
    specs = [F.parse_definition(d) for d in w.forces]
    c = rigid_constraints(w.system)
    m = w.system.mass
    E = lambda e, vel: e.lennard_jones + e.coulomb + integrate.kinetic_energy(m, vel)
    gains, kes, worst_bond = [], [], 0.0
    for k in range(4):
        topo = F.Topology(w.system)
        fs = [F.ForceFactory.make(topo, d, precision) for d in w.forces]
        lf = integrate.Leapfrog(topo, fs, w.system.positions, v * (1 + k * 1e-12), m, DT, constraints=c).initialize()
        lf.run(100)
        x100, v100, _, e100 = lf.state()
        if k == 0 and precision == "fp64":
            r0 = oracle.evaluate(w.system, specs)
            x, _, _, _ = oracle.leapfrog(w.system, specs, v, DT, 100, forces=r0["forces"], constraints=c)
            print(f"\nrigid water: |dx| at 100 steps {np.abs(x100 - x).max():.2e} A")
            assert np.abs(x100 - x).max() <= 1e-6
        lf.run(900)
        xg, vg, _, eg = lf.state()
        assert lf.constraint_limit_hits() == 0
        gains.append(E(eg, vg) - E(e100, v100))
        kes.append(integrate.kinetic_energy(m, vg))
        d = np.linalg.norm(xg[c["atoms"][:, 0]] - xg[c["atoms"][:, 1]], axis=1)
        worst_bond = max(worst_bond, float(np.abs(d - c["rest"]).max()))
        topo.close()
    print(f"rigid water {precision}: E(1000) - E(100) {' '.join(f'{g:+.1f}' for g in gains)} kcal/mol "
          f"(KE {np.mean(kes):.0f}), bond error {worst_bond:.2e} A")
    assert worst_bond <= 1e-3
    assert abs(np.mean(gains)) <= 0.02 * np.mean(kes)
