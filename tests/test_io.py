"""PSF / PAR / XYZ / PDB / configuration readers (protomol_b200.io) and the
System they build, restating frontend/buildTopology.cpp:

* round trips of the synthetic systems through the writers;
* the PAR dialects (CHARMM28 sections, X-PLOR records), NBFIX, wildcards;
* molecules as connected components numbered by their lowest atom;
* the reference's own example inputs, where the reference tree is present:
  the water box and the 14,281-atom BPTI configuration, whose nonbonded
  forces the restatement and the compiled reference then evaluate alike."""
import os

import numpy as np
import pytest

from protomol_b200 import forces as F
from protomol_b200 import io, systems
from protomol_b200.systems import SQRT_COULOMB_CONSTANT

from oracle.oracle import reference_root

REFERENCE = reference_root() or ""
EXAMPLES = os.path.join(REFERENCE, "examples")
needs_examples = pytest.mark.skipif(not os.path.isdir(EXAMPLES), reason="reference examples not present")

FIELDS = ("positions", "atom_type", "molecule", "mass", "type_params", "lj_table", "exclusions", "exclusion_check")


def _write(tmp_path, s):
    paths = [str(tmp_path / f"s.{ext}") for ext in ("psf", "par", "xyz")]
    io.write_psf(paths[0], s)
    io.write_par(paths[1], s)
    io.write_xyz(paths[2], s)
    return paths


@pytest.mark.parametrize("make", [systems.water_box_216, systems.vacuum_chain_104, systems.ionic_fluid_216])
def test_synthetic_systems_round_trip(tmp_path, make):
    s = make()
    t = io.load(*_write(tmp_path, s), s.box, s.cell_size, periodic=s.periodic)
    for f in FIELDS:
        if f in ("atom_type", "type_params", "lj_table"):
            continue
        assert np.array_equal(getattr(s, f), getattr(t, f)), f
    # types are renumbered in order of first appearance; the per-atom
    # parameters are the same
    assert np.array_equal(s.type_params[s.atom_type], t.type_params[t.atom_type])
    ia, ib = np.ix_(s.atom_type, s.atom_type), np.ix_(t.atom_type, t.atom_type)
    assert np.array_equal(s.lj_table[ia], t.lj_table[ib])
    assert t.n_types == len(np.unique(s.atom_type))
    # the file holds q = scaled / sqrt(332.0636); scaling back is within one rounding
    assert np.allclose(t.scaled_charge, s.scaled_charge, rtol=2.3e-16, atol=0)
    assert t.bonds == s.bonds and t.angles == s.angles and t.dihedrals == s.dihedrals


def test_nbfix_entries_round_trip(tmp_path):
    s = systems.water_box_216()
    s.lj_table[0, 1] = s.lj_table[1, 0] = (1.5e5, 600.0, 1.2e5, 500.0)
    paths = _write(tmp_path, s)
    assert "NBFIX" in open(paths[1]).read()
    t = io.load(*paths, s.box, s.cell_size)
    assert np.array_equal(t.lj_table, s.lj_table)


def test_molecules_are_components_numbered_by_lowest_atom():
    # atoms 5-6 bonded first in the list; 2-3-4 joined by an angle only;
    # 7-10 joined by a dihedral; 11 alone
    mol = io.molecules_of(12, [(5, 6), (0, 1)], [(2, 3, 4)], [(10, 8, 9, 7)], [])
    assert mol.tolist() == [0, 0, 1, 1, 1, 2, 2, 3, 3, 3, 3, 4]


def test_parameter_look_up_prefers_exact_names():
    pats = ["C*", "CT", "H%", "O#", "N+", "CA"]
    assert io.match_type(pats, "CT") == 1          # exact beats the earlier wildcard
    assert io.match_type(pats, "CB") == 0
    assert io.match_type(pats, "CA") == 5
    assert io.match_type(pats, "HA") == 2
    assert io.match_type(pats, "HAB") == -1        # % is one character
    assert io.match_type(pats, "O12") == 3 and io.match_type(pats, "O") == 3
    assert io.match_type(pats, "OX") == -1
    assert io.match_type(pats, "N3") == 4 and io.match_type(pats, "N33") == -1


def test_charmm28_and_xplor_dialects(tmp_path):
    c28 = tmp_path / "c28.par"
    c28.write_text(
        "* title\n*\nBONDS\nOT HT 450.0 0.9572\n\n"
        "NONBONDED nbxmod 5 atom cdiel shift vatom vdistance vswitch -\n"
        "cutnb 14.0 ctofnb 12.0 ctonnb 10.0 eps 1.0 e14fac 1.0 wmin 1.5\n"
        "OT 0.0 -0.1521 1.7682 ! water oxygen\n"
        "CT 0.0 -0.0800 2.0600 0.0 -0.0100 1.9000\n\n"
        "NBFIX\nOT CT 1000.0 20.0\n\nEND\n")
    p = io.read_par(str(c28))
    assert p["nonbonded"] == [("OT", 0.1521, 1.7682, 0.1521, 1.7682), ("CT", 0.08, 2.06, 0.01, 1.9)]
    assert p["nbfix"] == [("OT", "CT", 1000.0, 20.0, 1000.0, 20.0)]
    xp = tmp_path / "xplor.par"
    xp.write_text(" REMARKS water\n SET ECHO=FALSE END\n {a comment\n  across lines}\n"
                  " BOND  OT   HT       450.000 {SD=      .026}       .957\n"
                  " NONBONDED  OT       .1521   3.1506    .1521   3.1506 ! oxygen\n"
                  " NONBONDED  HT       .0460    .4000    .0460    .4000\n")
    p = io.read_par(str(xp))
    c = 2.0 ** (-5.0 / 6.0)
    assert p["nonbonded"] == [("OT", 0.1521, 3.1506 * c, 0.1521, 3.1506 * c), ("HT", 0.046, 0.4 * c, 0.046, 0.4 * c)]


def test_missing_parameters_raise(tmp_path):
    s = systems.water_box_216()
    psf, par, xyz = _write(tmp_path, s)
    open(par, "w").write("NONBONDED\nT0 0.0 -0.1 1.7\nEND\n")
    with pytest.raises(ValueError, match="T1"):
        io.load(psf, par, xyz, s.box, s.cell_size)


def test_conf_reader_joins_force_definitions(tmp_path):
    conf = tmp_path / "run.conf"
    conf.write_text("posfile s.xyz\npsffile s.psf\nparfile s.par\nexclude 1-4\n"
                    "boundaryConditions periodic\ncellBasisVector1 18.0 0 0\ncellBasisVector2 0 18.0 0\n"
                    "cellBasisVector3 0 0 18.0\ncellOrigin 0 0 0\ncellsize 5\n"
                    "Integrator {\n  level 0 Leapfrog {\n    timestep 1\n    force Bond\n"
                    "    Force time LennardJones -switchingFunction C2   # switched\n"
                    "      -algorithm NonbondedCutoff -switchon 8\n      -cutoff 9 -cutoff 9\n  }\n}\n")
    c = io.read_conf(str(conf))
    assert c["forces"] == ["Bond", "LennardJones -switchingFunction C2 -algorithm NonbondedCutoff -switchon 8 "
                                   "-cutoff 9 -cutoff 9"]
    assert c["exclude"] == "1-4" and c["cellbasisvector2"] == ["0", "18.0", "0"]
    s = systems.water_box_216()
    _write(tmp_path, s)
    t, fs = io.load_conf(str(conf))
    assert t.periodic and np.array_equal(t.box_lengths, [18.0, 18.0, 18.0]) and t.cell_size == 5.0
    assert np.array_equal(t.exclusions, systems.build_exclusions(s.bonds, s.angles, s.dihedrals, "1-4")[0])
    spec = F.parse_definition(fs[1])
    assert spec["kind"] == "cut" and spec["terms"][0][:2] == ("C2", "LennardJones")


@needs_examples
def test_reference_water_example():
    d = os.path.join(EXAMPLES, "water_648")
    s = io.load(os.path.join(d, "water648.tip3.psf"), os.path.join(d, "water648.tip3.par"),
                os.path.join(d, "water648.fluid.pos.xyz"), np.diag([18.6259267382819] * 3 + [0])[:, :3], 5.0)
    assert s.n_atoms == 648 and s.n_types == 2 and s.molecule.max() == 215
    assert s.scaled_charge[0] == -0.8476 * SQRT_COULOMB_CONSTANT
    assert np.isclose(s.type_params[0, 1], 3.1506 * 2.0 ** (-5.0 / 6.0), rtol=1e-15)
    assert s.exclusions.shape == (648, 3)          # O-H1, O-H2 bonds and the H1-H2 1-3 pair per water


@needs_examples
def test_reference_bpti_configuration():
    from oracle import oracle
    s, fs = io.load_conf(os.path.join(EXAMPLES, "bpti_water_14281", "bpti.pme.opt.conf"))
    assert s.n_atoms == 14281 and s.n_types == 26 and s.periodic
    assert np.array_equal(s.box_lengths, [63.0, 50.0, 50.0]) and s.cell_size == 6.0
    nonbonded = [d for d in fs if d.split()[0] in ("LennardJones", "Coulomb", "CoulombEwaldReal")]
    specs = [F.parse_definition(d) for d in nonbonded]
    assert [sp["kind"] for sp in specs] == ["cut", "pme"]
    if not oracle.reference_available():
        pytest.skip("oracle/_ref not built here")
    a = oracle.evaluate(s, specs)
    b = oracle.run_reference(s, specs)
    rms = np.sqrt((b["forces"] ** 2).sum(1).mean())
    assert np.abs(a["forces"] - b["forces"]).max() <= 1e-12 * rms
    assert abs(a["lennard_jones"] - b["lennard_jones"]) <= 1e-12 * abs(b["lennard_jones"])
    assert abs(a["coulomb"] - b["coulomb"]) <= 1e-9 * abs(b["coulomb"])


@needs_examples
def test_reference_example_force_lines_parse():
    """Every nonbonded force line of the reference's example configurations
    that uses this path's algorithms and switching functions parses (the
    factory ignores case); Cn switching, FullEwald and MultiGrid are not on
    this path."""
    import glob
    nonbonded = ("lennardjones", "coulomb", "coulombewaldreal", "lennardjonestable", "coulombtable",
                 "coulombewaldrealtable")
    other = ("cn", "cmpcncn", "fullewald", "multigrid", "coulombmultigriddirect", "coulombmultigriddirecttable")
    parsed = 0
    for conf in sorted(glob.glob(os.path.join(EXAMPLES, "**", "*.conf"), recursive=True)):
        for d in io.read_conf(conf)["forces"]:
            toks = [t.lower() for t in d.split()]
            if toks[0] not in nonbonded or any(t in other for t in toks):
                continue
            if "-switchingfunction" in toks and toks.count("-switchingfunction") > \
                    sum(t in nonbonded and t != "coulombewaldrealtable" for t in toks):
                continue      # a switching function the registered id does not carry
            spec = F.parse_definition(d)
            assert spec["kind"] in ("cut", "full", "pme"), (conf, d)
            parsed += 1
    assert parsed >= 40
