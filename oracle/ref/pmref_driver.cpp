// pmref_driver.cpp -- runs ProtoMol's OWN force classes on a system file.
//
// TEST INFRASTRUCTURE ONLY.  Linked against the reference's sources (built
// by oracle/ref/Makefile into oracle/_ref/pmref), this driver is the pinned
// oracle: it constructs the reference's Topology<Periodic, Cubic> (or
// Topology<Vacuum, Cubic>) from a system blob written by
// protomol_b200.systems.System.save, instantiates the reference templates
// NonbondedCutoffSystemForce<CubicCellManager, OneAtomPair[Two]<...>>,
// NonbondedPMEwaldSystemForce<..., BSpline, CutoffSwitchingFunction> and
// NonbondedSimpleFullSystemForce<...> exactly as
// factories/registerForceExemplarsCutoff.cpp, ...FastElectrostatic.cpp and
// ...SimpleFull.cpp register them, evaluates them in order into one force
// block and ScalarStructure (like ForceGroup::evaluateSystemForces), and
// writes forces, energies, virial and the per-atom cell assignment.
//
// usage: pmref <system.bin> <out.bin> <repeat> <force spec>...
//   force spec tokens:
//     cut  n sw1 pot1 on1 rc1 alpha1 [sw2 pot2 on2 rc2 alpha2] algo_cutoff
//     pme  real recip corr nx ny nz order cutoff accuracy alpha
//     full n sw1 pot1 on1 rc1 alpha1 [sw2 pot2 on2 rc2 alpha2]
//   sw: 0 Universal 1 Cutoff 2 C1 3 C2 4 Shift; pot: 1 LJ 2 Coulomb 3 EwaldReal
// With repeat > 1 the evaluation is repeated (after one untimed warm-up) and
// the mean wall time per evaluation is reported (the CPU baseline).
// PMREF_MOLVIR=1 turns on ScalarStructure::molecularVirial() with the
// molecule positions set by buildMolecularCenterOfMass (unit masses);
// the molecule count, their positions and the molecular virial are then
// appended to the output.  PMREF_NO_VIRIAL=1 turns ScalarStructure::virial()
// off.  PMREF_HESSIAN=<path> (vacuum systems) puts the forces into a
// ForceGroup, runs ProtoMol's own Hessian (integrators/Hessian.cpp:
// findForces, then evaluate without mass re-weighting) and writes the dense
// 3N x 3N matrix to <path> (its nonbonded part reads separate LennardJones
// and Coulomb forces: give them as two "full 1 ..." specs).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "Report.h"
// Grid.h names report/error unqualified (the reference .cpp files that
// include it declare this using-directive first).
using namespace ProtoMol::Report;
#include "Topology.h"
#include "PeriodicBoundaryConditions.h"
#include "VacuumBoundaryConditions.h"
#include "CubicCellManager.h"
#include "CellListEnumerator_periodicBoundaries.h"
#include "CellListEnumerator_standard.h"
#include "NonbondedCutoffSystemForce.h"
#include "NonbondedSimpleFullSystemForce.h"
#include "NonbondedPMEwaldSystemForce.h"
#include "OneAtomPair.h"
#include "OneAtomPairTwo.h"
#include "LennardJonesTableForce.h"
#include "CoulombTableForce.h"
#include "CoulombEwaldRealTableForce.h"
#include "LennardJonesForce.h"
#include "CoulombForce.h"
#include "CoulombEwaldRealForce.h"
#include "C1SwitchingFunction.h"
#include "C2SwitchingFunction.h"
#include "CutoffSwitchingFunction.h"
#include "ShiftSwitchingFunction.h"
#include "UniversalSwitchingFunction.h"
#include "BSpline.h"
#include "ScalarStructure.h"
#include "Vector3DBlock.h"
#include "topologyutilities.h"
#include "ForceGroup.h"
#include "Hessian.h"

using namespace ProtoMol;

typedef PeriodicBoundaryConditions PBC;
typedef VacuumBoundaryConditions VBC;
typedef Topology<PBC, CubicCellManager> PTopo;
typedef Topology<VBC, CubicCellManager> VTopo;

struct Blob {
    int n, t, e, periodic;
    double box[12], csf, cell;
    std::vector<double> pos, q, lj;
    std::vector<int> type, mol, excl, check;
};

static bool read_blob(const char* path, Blob& b)
{
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    char magic[8];
    bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, "PMSYS001", 8) == 0;
    int h[4];
    ok = ok && fread(h, sizeof(int), 4, f) == 4;
    b.n = h[0]; b.t = h[1]; b.e = h[2]; b.periodic = h[3];
    ok = ok && fread(b.box, sizeof(double), 12, f) == 12;
    double cc[2];
    ok = ok && fread(cc, sizeof(double), 2, f) == 2;
    b.csf = cc[0]; b.cell = cc[1];
    b.pos.resize(3 * (size_t)b.n); b.q.resize(b.n); b.type.resize(b.n); b.mol.resize(b.n);
    b.lj.resize(4 * (size_t)b.t * b.t); b.excl.resize(3 * (size_t)b.e); b.check.resize(b.e);
    ok = ok && fread(b.pos.data(), sizeof(double), b.pos.size(), f) == b.pos.size();
    ok = ok && fread(b.q.data(), sizeof(double), b.q.size(), f) == b.q.size();
    ok = ok && fread(b.type.data(), sizeof(int), b.type.size(), f) == b.type.size();
    ok = ok && fread(b.mol.data(), sizeof(int), b.mol.size(), f) == b.mol.size();
    ok = ok && fread(b.lj.data(), sizeof(double), b.lj.size(), f) == b.lj.size();
    ok = ok && (b.e == 0 || fread(b.excl.data(), sizeof(int), b.excl.size(), f) == b.excl.size());
    ok = ok && (b.e == 0 || fread(b.check.data(), sizeof(int), b.check.size(), f) == b.check.size());
    fclose(f);
    return ok;
}

// Fills the GenericTopology members the nonbonded forces read (the same
// members frontend/buildTopology.cpp fills from PSF/PAR).
static void fill_topology(GenericTopology* topo, const Blob& b)
{
    topo->atoms.resize(b.n);
    int nmol = 0;
    for (int i = 0; i < b.n; ++i) {
        topo->atoms[i].type = b.type[i];
        topo->atoms[i].scaledCharge = b.q[i];
        topo->atoms[i].scaledMass = 1.0;
        topo->atoms[i].molecule = b.mol[i];
        topo->atoms[i].cellListNext = -1;
        if (b.mol[i] + 1 > nmol) nmol = b.mol[i] + 1;
    }
    topo->molecules.resize(nmol);
    for (int i = 0; i < b.n; ++i) topo->molecules[b.mol[i]].atoms.push_back(i);
    topo->lennardJonesParameters.resize(b.t);
    for (int i = 0; i < b.t; ++i)
        for (int j = 0; j < b.t; ++j) {
            const double* p = &b.lj[4 * ((size_t)i * b.t + j)];
            LennardJonesParameters par;
            par.A = p[0]; par.B = p[1]; par.A14 = p[2]; par.B14 = p[3];
            topo->lennardJonesParameters.set(i, j, par);
        }
    topo->exclusions.resize(b.n);
    for (int k = 0; k < b.e; ++k)
        topo->exclusions.add(b.excl[3 * k], b.excl[3 * k + 1], (ExclusionClass)b.excl[3 * k + 2]);
    for (int k = 0; k < b.e; ++k)
        if (b.check[k] != b.excl[3 * k + 2])
            topo->exclusions.add(b.excl[3 * k], b.excl[3 * k + 1], (ExclusionClass)b.check[k]);
    topo->exclusions.optimize();
}

// ---------------------------------------------------------------- factories
struct Term { int sw, pot; double on, rc, alpha; };

template <class SW> SW make_sw(const Term& t);
template <> C1SwitchingFunction make_sw<C1SwitchingFunction>(const Term& t) { return C1SwitchingFunction(t.rc); }
template <> C2SwitchingFunction make_sw<C2SwitchingFunction>(const Term& t) { return C2SwitchingFunction(t.on, t.rc); }
template <> CutoffSwitchingFunction make_sw<CutoffSwitchingFunction>(const Term& t) { return CutoffSwitchingFunction(t.rc); }
template <> ShiftSwitchingFunction make_sw<ShiftSwitchingFunction>(const Term& t) { return ShiftSwitchingFunction(t.rc); }
template <> UniversalSwitchingFunction make_sw<UniversalSwitchingFunction>(const Term&) { return UniversalSwitchingFunction(); }

template <class P> P make_pot(const Term& t);
template <> LennardJonesForce make_pot<LennardJonesForce>(const Term&) { return LennardJonesForce(); }
template <> CoulombForce make_pot<CoulombForce>(const Term&) { return CoulombForce(); }
template <> CoulombEwaldRealForce make_pot<CoulombEwaldRealForce>(const Term& t) { return CoulombEwaldRealForce(t.alpha); }

// the registered look-up-table potentials (factories/registerForceExemplarsCutoff.cpp:47-48,58,69):
// the term's switching function is the tabulated one; the pair applies Universal
typedef LennardJonesTableForce<C2SwitchingFunction, 7, Real> LJTableC2;
typedef CoulombTableForce<CutoffSwitchingFunction, 6, Real> CoulombTableCutoff;
typedef CoulombTableForce<ShiftSwitchingFunction, 6, Real> CoulombTableShift;
typedef CoulombEwaldRealTableForce<CutoffSwitchingFunction, 6, Real> EwaldRealTableCutoff;
template <> LJTableC2 make_pot<LJTableC2>(const Term& t) { return LJTableC2(C2SwitchingFunction(t.on, t.rc)); }
template <> CoulombTableCutoff make_pot<CoulombTableCutoff>(const Term& t) { return CoulombTableCutoff(CutoffSwitchingFunction(t.rc)); }
template <> CoulombTableShift make_pot<CoulombTableShift>(const Term& t) { return CoulombTableShift(ShiftSwitchingFunction(t.rc)); }
template <> EwaldRealTableCutoff make_pot<EwaldRealTableCutoff>(const Term& t)
{
    return EwaldRealTableCutoff(CutoffSwitchingFunction(t.rc), t.alpha);
}

template <class SW1, class P1>
static SystemForce* cut1(const Term& a, double algo)
{
    typedef OneAtomPair<PBC, SW1, P1> OAP;
    return new NonbondedCutoffSystemForce<CubicCellManager, OAP>(algo, OAP(make_pot<P1>(a), make_sw<SW1>(a)));
}

template <class SW1, class P1, class SW2, class P2>
static SystemForce* cut2(const Term& a, const Term& b, double algo)
{
    typedef OneAtomPairTwo<PBC, SW1, P1, SW2, P2> OAP;
    return new NonbondedCutoffSystemForce<CubicCellManager, OAP>(
        algo, OAP(make_pot<P1>(a), make_sw<SW1>(a), make_pot<P2>(b), make_sw<SW2>(b)));
}

template <class SW1, class P1, class SW2, class P2>
static SystemForce* full2(const Term& a, const Term& b)
{
    typedef OneAtomPairTwo<VBC, SW1, P1, SW2, P2> OAP;
    return new NonbondedSimpleFullSystemForce<OAP>(OAP(make_pot<P1>(a), make_sw<SW1>(a), make_pot<P2>(b), make_sw<SW2>(b)), 64);
}

#define SWC(x) x##SwitchingFunction
static SystemForce* make_cut(const std::vector<Term>& t, double algo)
{
    if (t.size() == 1) {
        const Term& a = t[0];
#define ONE(S, P, SWID, POTID) if (a.sw == SWID && a.pot == POTID) return cut1<SWC(S), P>(a, algo);
        ONE(C1, CoulombForce, 2, 2) ONE(C2, CoulombForce, 3, 2) ONE(Cutoff, CoulombForce, 1, 2)
        ONE(Shift, CoulombForce, 4, 2) ONE(Cutoff, CoulombEwaldRealForce, 1, 3)
        ONE(C1, LennardJonesForce, 2, 1) ONE(C2, LennardJonesForce, 3, 1)
        ONE(Cutoff, LennardJonesForce, 1, 1) ONE(Shift, LennardJonesForce, 4, 1)
        // table potentials: pot 4 LennardJonesTable, 5 CoulombTable, 6 CoulombEwaldRealTable
        ONE(Universal, LJTableC2, 3, 4) ONE(Universal, CoulombTableCutoff, 1, 5)
        ONE(Universal, CoulombTableShift, 4, 5) ONE(Universal, EwaldRealTableCutoff, 1, 6)
#undef ONE
    } else if (t.size() == 2) {
        const Term& a = t[0];
        const Term& b = t[1];
#define TWO(S1, S2, P2, SWID1, SWID2, POTID2) \
        if (a.sw == SWID1 && a.pot == 1 && b.sw == SWID2 && b.pot == POTID2) \
            return cut2<SWC(S1), LennardJonesForce, SWC(S2), P2>(a, b, algo);
        TWO(C1, Cutoff, CoulombEwaldRealForce, 2, 1, 3) TWO(C1, Shift, CoulombForce, 2, 4, 2)
        TWO(C2, C1, CoulombForce, 3, 2, 2) TWO(C2, Cutoff, CoulombEwaldRealForce, 3, 1, 3)
        TWO(C2, Cutoff, CoulombForce, 3, 1, 2) TWO(C2, Shift, CoulombForce, 3, 4, 2)
        TWO(Cutoff, Cutoff, CoulombEwaldRealForce, 1, 1, 3) TWO(C2, C2, CoulombForce, 3, 3, 2)
        // LennardJones + CoulombEwaldRealTable (registerForceExemplarsCutoff.cpp:86,101,132)
        if (a.pot == 1 && b.pot == 6 && b.sw == 1) {
            if (a.sw == 2) return cut2<SWC(C1), LennardJonesForce, SWC(Universal), EwaldRealTableCutoff>(a, b, algo);
            if (a.sw == 3) return cut2<SWC(C2), LennardJonesForce, SWC(Universal), EwaldRealTableCutoff>(a, b, algo);
            if (a.sw == 1) return cut2<SWC(Cutoff), LennardJonesForce, SWC(Universal), EwaldRealTableCutoff>(a, b, algo);
        }
        // LennardJonesTable + CoulombEwaldRealTable / CoulombTable (:133-134)
        if (a.pot == 4 && a.sw == 3 && b.pot == 6 && b.sw == 1)
            return cut2<SWC(Universal), LJTableC2, SWC(Universal), EwaldRealTableCutoff>(a, b, algo);
        if (a.pot == 4 && a.sw == 3 && b.pot == 5 && b.sw == 4)
            return cut2<SWC(Universal), LJTableC2, SWC(Universal), CoulombTableShift>(a, b, algo);
#undef TWO
    }
    return NULL;
}

template <class SW, class P>
static SystemForce* full1(const Term& a)
{
    typedef OneAtomPair<VBC, SW, P> OAP;
    return new NonbondedSimpleFullSystemForce<OAP>(OAP(make_pot<P>(a), make_sw<SW>(a)), 64);
}

static SystemForce* make_full(const std::vector<Term>& t)
{
    // one term (registerForceExemplarsSimpleFull.cpp): LennardJones or
    // Coulomb under Universal, C1 or C2
    if (t.size() == 1 && (t[0].pot == 1 || t[0].pot == 2)) {
        const bool lj = t[0].pot == 1;
        if (t[0].sw == 0) return lj ? full1<UniversalSwitchingFunction, LennardJonesForce>(t[0])
                                    : full1<UniversalSwitchingFunction, CoulombForce>(t[0]);
        if (t[0].sw == 2) return lj ? full1<C1SwitchingFunction, LennardJonesForce>(t[0])
                                    : full1<C1SwitchingFunction, CoulombForce>(t[0]);
        if (t[0].sw == 3) return lj ? full1<C2SwitchingFunction, LennardJonesForce>(t[0])
                                    : full1<C2SwitchingFunction, CoulombForce>(t[0]);
    }
    if (t.size() == 2 && t[0].pot == 1 && t[1].pot == 2) {
        if (t[0].sw == 0 && t[1].sw == 0)
            return full2<UniversalSwitchingFunction, LennardJonesForce, UniversalSwitchingFunction, CoulombForce>(t[0], t[1]);
        if (t[0].sw == 3 && t[1].sw == 3)
            return full2<C2SwitchingFunction, LennardJonesForce, C2SwitchingFunction, CoulombForce>(t[0], t[1]);
    }
    return NULL;
}

static SystemForce* make_pme(int real, int recip, int corr, int nx, int ny, int nz, int order,
                             double cutoff, double acc, double alpha)
{
#define PME(a, b, c) if (real == a && recip == b && corr == c) \
    return new NonbondedPMEwaldSystemForce<PBC, CubicCellManager, a, b, c, BSpline, CutoffSwitchingFunction>( \
        nx, ny, nz, order, cutoff, acc, alpha, 3.0);
    PME(1, 1, 1) PME(1, 0, 0) PME(1, 0, 1) PME(0, 1, 0) PME(0, 1, 1) PME(0, 0, 1) PME(1, 1, 0)
#undef PME
    return NULL;
}

static double now()
{
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int main(int argc, char** argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: pmref <system.bin> <out.bin> <repeat> <force spec>...\n");
        return 2;
    }
    Blob b;
    if (!read_blob(argv[1], b)) { fprintf(stderr, "pmref: cannot read %s\n", argv[1]); return 2; }
    int repeat = atoi(argv[3]);
    std::vector<SystemForce*> forces;
    int a = 4;
    while (a < argc) {
        std::string kind = argv[a++];
        if (kind == "cut" || kind == "full") {
            int n = atoi(argv[a++]);
            std::vector<Term> t(n);
            for (int k = 0; k < n; ++k) {
                t[k].sw = atoi(argv[a++]); t[k].pot = atoi(argv[a++]);
                t[k].on = atof(argv[a++]); t[k].rc = atof(argv[a++]); t[k].alpha = atof(argv[a++]);
            }
            SystemForce* f = kind == "cut" ? make_cut(t, atof(argv[a++])) : make_full(t);
            if (!f) { fprintf(stderr, "pmref: unsupported force combination\n"); return 3; }
            forces.push_back(f);
        } else if (kind == "pme") {
            int v[7];
            for (int k = 0; k < 7; ++k) v[k] = atoi(argv[a++]);
            double cutoff = atof(argv[a++]), acc = atof(argv[a++]), alpha = atof(argv[a++]);
            SystemForce* f = make_pme(v[0], v[1], v[2], v[3], v[4], v[5], v[6], cutoff, acc, alpha);
            if (!f) { fprintf(stderr, "pmref: unsupported PME combination\n"); return 3; }
            forces.push_back(f);
        } else {
            fprintf(stderr, "pmref: unknown force kind %s\n", kind.c_str());
            return 2;
        }
    }

    Vector3D e1(b.box[0], b.box[1], b.box[2]), e2(b.box[3], b.box[4], b.box[5]),
        e3(b.box[6], b.box[7], b.box[8]), o(b.box[9], b.box[10], b.box[11]);
    GenericTopology* topo;
    if (b.periodic)
        topo = new PTopo(b.csf, ExclusionType(ExclusionType::ONE4MODIFIED), PBC(e1, e2, e3, o), CubicCellManager(b.cell));
    else
        topo = new VTopo(b.csf, ExclusionType(ExclusionType::ONE4MODIFIED), VBC(), CubicCellManager(b.cell));
    fill_topology(topo, b);

    Vector3DBlock pos(b.n), frc(b.n);
    for (int i = 0; i < b.n; ++i) pos[i] = Vector3D(b.pos[3 * i], b.pos[3 * i + 1], b.pos[3 * i + 2]);
    ScalarStructure en;
    const char* mv_env = getenv("PMREF_MOLVIR");
    const char* nv_env = getenv("PMREF_NO_VIRIAL");
    const bool molvir = mv_env && atoi(mv_env) != 0;
    en.molecularVirial(molvir);
    en.virial(!(nv_env && atoi(nv_env) != 0));
    if (molvir) buildMolecularCenterOfMass(&pos, topo);

    double t0 = 0.0, t1 = 0.0;
    int reps = repeat > 1 ? repeat + 1 : 1;
    for (int r = 0; r < reps; ++r) {
        if (r == 1) t0 = now();
        frc.zero();
        en.clear();
        topo->uncacheCellList();
        for (size_t k = 0; k < forces.size(); ++k) forces[k]->evaluate(topo, &pos, &frc, &en);
    }
    t1 = now();
    double per_eval = repeat > 1 ? (t1 - t0) / repeat : 0.0;

    std::vector<int> cells(3 * (size_t)b.n, 0);
    int dims[3] = {0, 0, 0};
    if (b.periodic) {
        PTopo* pt = (PTopo*)topo;
        pt->uncacheCellList();
        pt->updateCellLists(&pos);
        Vector3D delta(pt->boundaryConditions.origin() - pt->min);
        for (int i = 0; i < b.n; ++i) {
            CubicCellManager::Cell c = pt->cellManager.findCell(delta + pt->boundaryConditions.minimalPosition(pos[i]));
            cells[3 * i] = c.x; cells[3 * i + 1] = c.y; cells[3 * i + 2] = c.z;
        }
        dims[0] = pt->cellLists.getDimX(); dims[1] = pt->cellLists.getDimY(); dims[2] = pt->cellLists.getDimZ();
    }

    const char* hess_env = getenv("PMREF_HESSIAN");
    if (hess_env && !b.periodic) {
        // the group owns nothing here: it is never destroyed
        ForceGroup* fg = new ForceGroup();
        for (size_t k = 0; k < forces.size(); ++k) fg->addSystemForce(forces[k]);
        const unsigned int sz = 3 * (unsigned int)b.n;
        Hessian hess(sz);
        hess.clear();
        hess.findForces(fg);
        hess.evaluate(&pos, topo, false);
        FILE* hf = fopen(hess_env, "wb");
        if (!hf) return 4;
        fwrite(hess.hessM, sizeof(double), (size_t)sz * sz, hf);
        fclose(hf);
    }

    FILE* out = fopen(argv[2], "wb");
    if (!out) return 4;
    double hdr[13];
    hdr[0] = en[ScalarStructure::LENNARDJONES];
    hdr[1] = en[ScalarStructure::COULOMB];
    const int vslots[9] = {ScalarStructure::VIRIALXX, ScalarStructure::VIRIALXY, ScalarStructure::VIRIALXZ,
                           ScalarStructure::VIRIALYX, ScalarStructure::VIRIALYY, ScalarStructure::VIRIALYZ,
                           ScalarStructure::VIRIALZX, ScalarStructure::VIRIALZY, ScalarStructure::VIRIALZZ};
    for (int k = 0; k < 9; ++k) hdr[2 + k] = en[(ScalarStructure::Index)vslots[k]];
    hdr[11] = per_eval;
    hdr[12] = (double)repeat;
    fwrite(hdr, sizeof(double), 13, out);
    for (int i = 0; i < b.n; ++i) {
        double f3[3] = {frc[i].x, frc[i].y, frc[i].z};
        fwrite(f3, sizeof(double), 3, out);
    }
    fwrite(dims, sizeof(int), 3, out);
    fwrite(cells.data(), sizeof(int), cells.size(), out);
    if (molvir) {
        int nm = (int)topo->molecules.size();
        fwrite(&nm, sizeof(int), 1, out);
        for (int m = 0; m < nm; ++m) {
            const Vector3D& c = topo->molecules[m].position;
            double c3[3] = {c.x, c.y, c.z};
            fwrite(c3, sizeof(double), 3, out);
        }
        const int mslots[9] = {ScalarStructure::MOLVIRIALXX, ScalarStructure::MOLVIRIALXY,
                               ScalarStructure::MOLVIRIALXZ, ScalarStructure::MOLVIRIALYX,
                               ScalarStructure::MOLVIRIALYY, ScalarStructure::MOLVIRIALYZ,
                               ScalarStructure::MOLVIRIALZX, ScalarStructure::MOLVIRIALZY,
                               ScalarStructure::MOLVIRIALZZ};
        double mv[9];
        for (int k = 0; k < 9; ++k) mv[k] = en[(ScalarStructure::Index)mslots[k]];
        fwrite(mv, sizeof(double), 9, out);
    }
    fclose(out);
    for (size_t k = 0; k < forces.size(); ++k) delete forces[k];
    delete topo;
    return 0;
}
