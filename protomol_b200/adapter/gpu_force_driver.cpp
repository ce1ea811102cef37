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
// GPU_DRIVER_MOLVIR=1 turns ScalarStructure::molecularVirial() on, with the
// molecule positions from buildMolecularCenterOfMass (unit masses), and
// appends the molecular virial to the output.
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
#include "blob_topology.h"
#include "topologyutilities.h"

using namespace ProtoMol;

int main(int argc, char** argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: gpu_force_driver <system.bin> <out.bin> <repeat> <definition>...\n");
        return 2;
    }
    Blob b;
    if (!read_blob(argv[1], b) || !b.periodic) { fprintf(stderr, "bad system file\n"); return 2; }
    int repeat = atoi(argv[3]);
    Topology<PeriodicBoundaryConditions, CubicCellManager>& topo = *build_topology(b);
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
    const char* mv_env = getenv("GPU_DRIVER_MOLVIR");
    const bool molvir = mv_env && atoi(mv_env) != 0;
    en.molecularVirial(molvir);
    en.virial(true);
    if (molvir) buildMolecularCenterOfMass(&pos, &topo);
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
    if (molvir) {
        const ScalarStructure::Index m[9] = {
            ScalarStructure::MOLVIRIALXX, ScalarStructure::MOLVIRIALXY, ScalarStructure::MOLVIRIALXZ,
            ScalarStructure::MOLVIRIALYX, ScalarStructure::MOLVIRIALYY, ScalarStructure::MOLVIRIALYZ,
            ScalarStructure::MOLVIRIALZX, ScalarStructure::MOLVIRIALZY, ScalarStructure::MOLVIRIALZZ};
        double mv[9];
        for (int k = 0; k < 9; ++k) mv[k] = en[m[k]];
        fwrite(mv, sizeof(double), 9, out);
    }
    for (size_t k = 0; k < forces.size(); ++k) {
        std::string id = forces[k]->getIdNoAlias();
        fprintf(stderr, "made: %s\n", id.c_str());
        delete forces[k];
    }
    fclose(out);
    return 0;
}
