// gpu_force_driver.cpp -- evaluates GPU forces made by ProtoMol's own
// ForceFactory from force-definition strings (the drop-in path end to end).
//
// Builds the reference Topology<PeriodicBoundaryConditions, CubicCellManager>
// from a system blob (protomol_b200.systems.System.save), calls
// registerGpuForceExemplars(), makes every force with
// ForceFactory::make(errMsg, "<definition>") -- the reference's keyword
// parser (frontend/ForceFactoryDetails.cpp:48-293) -- evaluates them in order
// into one Vector3DBlock / ScalarStructure, like ForceGroup does, and writes
// energies, virial, forces and the per-evaluation wall time.
//
// usage: gpu_force_driver <system.bin> <out.bin> <repeat> <definition>...
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "Report.h"
using namespace ProtoMol::Report;
#include "CubicCellManager.h"
#include "ForceFactory.h"
#include "GpuNonbondedForce.h"
#include "PeriodicBoundaryConditions.h"
#include "ScalarStructure.h"
#include "SystemForce.h"
#include "Topology.h"
#include "Vector3DBlock.h"

using namespace ProtoMol;

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

int main(int argc, char** argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: gpu_force_driver <system.bin> <out.bin> <repeat> <definition>...\n");
        return 2;
    }
    Blob b;
    if (!read_blob(argv[1], b) || !b.periodic) { fprintf(stderr, "bad system file\n"); return 2; }
    int repeat = atoi(argv[3]);
    Vector3D e1(b.box[0], b.box[1], b.box[2]), e2(b.box[3], b.box[4], b.box[5]),
        e3(b.box[6], b.box[7], b.box[8]), o(b.box[9], b.box[10], b.box[11]);
    Topology<PeriodicBoundaryConditions, CubicCellManager> topo(
        b.csf, ExclusionType(ExclusionType::ONE4MODIFIED), PeriodicBoundaryConditions(e1, e2, e3, o),
        CubicCellManager(b.cell));
    // the GenericTopology members buildTopology fills (frontend/buildTopology.cpp)
    topo.atoms.resize(b.n);
    int nmol = 0;
    for (int i = 0; i < b.n; ++i) {
        topo.atoms[i].type = b.type[i];
        topo.atoms[i].scaledCharge = b.q[i];
        topo.atoms[i].scaledMass = 1.0;
        topo.atoms[i].molecule = b.mol[i];
        if (b.mol[i] + 1 > nmol) nmol = b.mol[i] + 1;
    }
    topo.molecules.resize(nmol);
    for (int i = 0; i < b.n; ++i) topo.molecules[b.mol[i]].atoms.push_back(i);
    topo.lennardJonesParameters.resize(b.t);
    for (int i = 0; i < b.t; ++i)
        for (int j = 0; j < b.t; ++j) {
            const double* p = &b.lj[4 * ((size_t)i * b.t + j)];
            LennardJonesParameters par;
            par.A = p[0]; par.B = p[1]; par.A14 = p[2]; par.B14 = p[3];
            topo.lennardJonesParameters.set(i, j, par);
        }
    topo.exclusions.resize(b.n);
    for (int k = 0; k < b.e; ++k)
        topo.exclusions.add(b.excl[3 * k], b.excl[3 * k + 1], (ExclusionClass)b.excl[3 * k + 2]);
    for (int k = 0; k < b.e; ++k)
        if (b.check[k] != b.excl[3 * k + 2])
            topo.exclusions.add(b.excl[3 * k], b.excl[3 * k + 1], (ExclusionClass)b.check[k]);
    topo.exclusions.optimize();

    registerGpuForceExemplars();
    std::vector<SystemForce*> forces;
    for (int a = 4; a < argc; ++a) {
        std::string err;
        Force* f = ForceFactory::make(err, argv[a], std::vector<Value>());
        SystemForce* sf = dynamic_cast<SystemForce*>(f);
        if (!sf) {
            fprintf(stderr, "ForceFactory could not make '%s': %s\n", argv[a], err.c_str());
            return 3;
        }
        forces.push_back(sf);
    }
    Vector3DBlock pos(b.n), frc(b.n);
    for (int i = 0; i < b.n; ++i) pos[i] = Vector3D(b.pos[3 * i], b.pos[3 * i + 1], b.pos[3 * i + 2]);
    ScalarStructure en;
    en.molecularVirial(false);
    en.virial(true);
    timespec t0, t1;
    int reps = repeat > 1 ? repeat + 1 : 1;
    for (int r = 0; r < reps; ++r) {
        if (r == 1) clock_gettime(CLOCK_MONOTONIC, &t0);
        frc.zero();
        en.clear();
        for (size_t k = 0; k < forces.size(); ++k) forces[k]->evaluate(&topo, &pos, &frc, &en);
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    double per = repeat > 1 ? ((t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec)) / repeat : 0.0;

    FILE* out = fopen(argv[2], "wb");
    if (!out) return 4;
    double hdr[13];
    hdr[0] = en[ScalarStructure::LENNARDJONES];
    hdr[1] = en[ScalarStructure::COULOMB];
    const ScalarStructure::Index v[9] = {ScalarStructure::VIRIALXX, ScalarStructure::VIRIALXY, ScalarStructure::VIRIALXZ,
                                         ScalarStructure::VIRIALYX, ScalarStructure::VIRIALYY, ScalarStructure::VIRIALYZ,
                                         ScalarStructure::VIRIALZX, ScalarStructure::VIRIALZY, ScalarStructure::VIRIALZZ};
    for (int k = 0; k < 9; ++k) hdr[2 + k] = en[v[k]];
    hdr[11] = per;
    hdr[12] = (double)repeat;
    fwrite(hdr, sizeof(double), 13, out);
    for (int i = 0; i < b.n; ++i) {
        double f3[3] = {frc[i].x, frc[i].y, frc[i].z};
        fwrite(f3, sizeof(double), 3, out);
    }
    for (size_t k = 0; k < forces.size(); ++k) {
        std::string id = forces[k]->getIdNoAlias();
        fprintf(stderr, "made: %s\n", id.c_str());
        delete forces[k];
    }
    fclose(out);
    return 0;
}
