"""The drop-in path end to end: GPU forces made by ProtoMol's OWN
ForceFactory from force-definition strings (protomol_b200/adapter:
GpuNonbondedForce + registerGpuForceExemplars, linked with the reference's
framework objects), evaluated through SystemForce::evaluate into a
Vector3DBlock / ScalarStructure, compared with the oracle."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import oracle
from protomol_b200 import forces as F
from protomol_b200 import systems, workloads

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "protomol_b200", "adapter", "_build", "gpu_force_driver")


def run_driver(system, defs, precision="mixed", repeat=1, molecular_virial=False):
    if not os.path.exists(DRIVER):
        pytest.skip("drop-in driver not built (needs the ProtoMol sources at build time)")
    env = dict(os.environ, PMGPU_PRECISION=precision, GPU_DRIVER_MOLVIR="1" if molecular_virial else "0")
    with tempfile.TemporaryDirectory() as td:
        sp, op = os.path.join(td, "s.bin"), os.path.join(td, "o.bin")
        system.save(sp)
        p = subprocess.run([DRIVER, sp, op, str(repeat), *defs], env=env, capture_output=True, text=True,
                           timeout=300)
        assert p.returncode == 0, p.stderr
        raw = open(op, "rb").read()
    n = system.n_atoms
    hdr = np.frombuffer(raw[:104], np.float64)
    f = np.frombuffer(raw[104:104 + 24 * n], np.float64).reshape(n, 3)
    made = [line[6:] for line in p.stderr.splitlines() if line.startswith("made: ")]
    out = {"lennard_jones": hdr[0], "coulomb": hdr[1], "virial": hdr[2:11], "forces": f,
           "seconds": hdr[11], "made": made}
    if molecular_virial:
        out["mol_virial"] = np.frombuffer(raw[104 + 24 * n:104 + 24 * n + 72], np.float64)
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["water216", "chain14281", "chain14281_pme_full"])
def test_force_factory_keywords_run_on_the_gpu(case, precision):
    w = workloads.water216() if case == "water216" else workloads.chain14281()
    system, defs = w.system, w.forces
    if case == "chain14281_pme_full":
        # LJ cutoff force + the whole PME force (-real -reciprocal -correction)
        defs = ["LennardJones -switchingFunction C2 -algorithm NonbondedCutoff -switchon 10 -cutoff 12 -cutoff 12",
                "Coulomb -algorithm PMEwald -real -reciprocal -correction -interpolation BSpline "
                "-gridsize 64 64 64 -cutoff 12 -order 4 -alpha 0.32"]
    r = run_driver(system, defs, precision)
    ref = oracle.evaluate(system, [F.parse_definition(d) for d in defs])
    # the factory matched the reference ids (same strings as the reference)
    for d, made in zip(defs, r["made"]):
        assert made.split()[0] == d.split()[0]
        assert "-algorithm" in made
    err = np.sqrt(((r["forces"] - ref["forces"]) ** 2).sum() / (ref["forces"] ** 2).sum())
    scale = abs(ref["lennard_jones"]) + abs(ref["coulomb"])
    tol_f, tol_e = (1e-9, 1e-10) if precision == "fp64" else (1e-5, 2e-6)
    assert err <= tol_f
    assert abs(r["lennard_jones"] + r["coulomb"] - ref["lennard_jones"] - ref["coulomb"]) <= tol_e * scale


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_molecular_virial_through_the_adapter(precision):
    """ScalarStructure::molecularVirial() on, the molecule positions set by
    ProtoMol's buildMolecularCenterOfMass in the driver: the adapter hands
    them to the GPU and fills the MOLVIRIAL slots."""
    system = systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)
    defs = ["LennardJones -switchingFunction C2 -algorithm NonbondedCutoff -switchon 8 -cutoff 9 -cutoff 9",
            "Coulomb -algorithm PMEwald -real -reciprocal -correction -interpolation BSpline "
            "-gridsize 24 24 24 -cutoff 9 -alpha 0.35"]
    r = run_driver(system, defs, precision, molecular_virial=True)
    ref = oracle.evaluate(system, [F.parse_definition(d) for d in defs], mol_pos=oracle.molecular_centers(system))
    d = np.abs(r["mol_virial"] - ref["mol_virial"]).max() / np.abs(ref["mol_virial"]).max()
    assert d <= (1e-10 if precision == "fp64" else 1e-6)


TABLE_DEFS = [
    "LennardJonesTable -switchingFunction C2 -algorithm NonbondedCutoff -switchon 7 -cutoff 9 -cutoff 9",
    "CoulombTable -switchingFunction Shift -algorithm NonbondedCutoff -cutoff 9 -cutoff 9",
    "CoulombEwaldRealTable -algorithm NonbondedCutoff -cutoff 9 -alpha 0.35 -cutoff 9",
    "LennardJones CoulombEwaldRealTable -switchingFunction C2 -algorithm NonbondedCutoff -switchon 7 -cutoff 10 "
    "-cutoff 8.5 -alpha 0.35 -cutoff 10",
    "LennardJonesTable CoulombTable -switchingFunction C2 -switchingFunction Shift -algorithm NonbondedCutoff "
    "-switchon 1 -cutoff 9 -cutoff 9.5 -cutoff 9.5",
]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("definition", TABLE_DEFS)
def test_table_force_keywords_run_on_the_gpu(definition, precision):
    """Table potentials made by ProtoMol's ForceFactory from their own ids."""
    system = systems.chain_in_water(n_chain=60, n_water=400, length=24.0, seed=11)
    r = run_driver(system, [definition], precision)
    ref = oracle.evaluate(system, [F.parse_definition(definition)])
    assert r["made"][0] == F.cutoff_ident(F.parse_definition(definition)["terms"])
    err = np.sqrt(((r["forces"] - ref["forces"]) ** 2).sum() / (ref["forces"] ** 2).sum())
    scale = abs(ref["lennard_jones"]) + abs(ref["coulomb"])
    tol_f, tol_e = (1e-9, 1e-10) if precision == "fp64" else (1e-5, 2e-6)
    assert err <= tol_f
    assert abs(r["lennard_jones"] + r["coulomb"] - ref["lennard_jones"] - ref["coulomb"]) <= tol_e * scale


LEAPFROG = os.path.join(ROOT, "protomol_b200", "adapter", "_build", "gpu_leapfrog_driver")


def run_leapfrog(system, velocities, defs, steps, mode, precision="mixed"):
    if not os.path.exists(LEAPFROG):
        pytest.skip("drop-in driver not built (needs the ProtoMol sources at build time)")
    env = dict(os.environ, PMGPU_PRECISION=precision)
    with tempfile.TemporaryDirectory() as td:
        sp, dp, op = (os.path.join(td, f) for f in ("s.bin", "d.bin", "o.bin"))
        system.save(sp)
        np.concatenate([system.mass, velocities.ravel()]).astype(np.float64).tofile(dp)
        p = subprocess.run([LEAPFROG, sp, dp, op, str(steps), "1.0", mode, *defs], env=env, capture_output=True,
                           text=True, timeout=600)
        assert p.returncode == 0, p.stderr
        raw = np.fromfile(op)
    n = system.n_atoms
    calls = [int(line.split()[-1]) for line in p.stderr.splitlines() if line.startswith("gpu evaluations:")]
    return {"epot": raw[0], "ekin": raw[1], "positions": raw[2:2 + 3 * n].reshape(n, 3),
            "velocities": raw[2 + 3 * n:].reshape(n, 3), "gpu_calls": calls[0] if calls else None}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_reference_leapfrog_integrator_runs_on_the_gpu_forces(precision):
    """ProtoMol's own LeapfrogIntegrator and ForceGroup, 20 steps of 1 fs on
    a 216-particle ionic Lennard-Jones fluid with the split Ewald real-space
    force and PME (two GPU forces in one group), against the same run on the
    reference forces the GPU ones wrap.  The group's two GPU forces run as
    one pmgpu_evaluate per step once the group is learned (first step)."""
    from protomol_b200 import integrate
    s = systems.ionic_fluid_216()
    alpha = systems.ewald_alpha(9.0)
    defs = [workloads.lj_ewald_split(8, 9, alpha), workloads.pme_reciprocal((20, 20, 20), 9, alpha)]
    v = integrate.maxwell_boltzmann(s.mass, 300.0, seed=7)
    steps = 20
    cpu = run_leapfrog(s, v, defs, steps, "cpu")
    gpu = run_leapfrog(s, v, defs, steps, "gpu", precision)
    dx = np.abs(gpu["positions"] - cpu["positions"]).max()
    dv = np.abs(gpu["velocities"] - cpu["velocities"]).max()
    print(f"\n{precision}: 20 Leapfrog steps, max |dx| {dx:.2e} A, max |dv| {dv:.2e}, "
          f"E_pot {gpu['epot']:.6f} / {cpu['epot']:.6f}, GPU calls {gpu['gpu_calls']}")
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert dx <= tol
    assert abs(gpu["epot"] - cpu["epot"]) <= (1e-9 if precision == "fp64" else 1e-6) * abs(cpu["epot"])
    # initializeForces + 20 steps = 21 group evaluations: the first one learns
    # the group (one call per force), the other 20 make one call each
    assert gpu["gpu_calls"] == 2 + steps
