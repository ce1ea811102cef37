// gpu_leapfrog_driver.cpp -- runs ProtoMol's own LeapfrogIntegrator
// (integrators/LeapfrogIntegrator.cpp) over a ForceGroup of nonbonded forces
// made by ProtoMol's ForceFactory, on the GPU forces of the drop-in
// (registerGpuForceExemplars) or on the reference forces they wrap, so that
// the two trajectories can be compared: the unchanged integrator,
// ForceGroup::evaluateSystemForces and Vector3DBlock / ScalarStructure on
// both sides, only the force objects differ.
//
// usage: gpu_leapfrog_driver <system.bin> <dynamics.bin> <out.bin> <steps> <timestep fs> <gpu|cpu> <definition>...
//   dynamics.bin: N masses, then 3N velocities (doubles, A / fs units of ProtoMol)
//   out.bin: potential energy, kinetic energy after the run, then 3N positions, 3N velocities
// LF_CONSTRAINTS=<file> adds the topology's bonds and angles and ProtoMol's
// SHAKE / RATTLE modifiers as protomol.cpp:553-577 attaches them; the text
// file holds "n_bonds n_angles shake_eps shake_max_iter rattle_eps
// rattle_max_iter", then n_bonds lines "a1 a2 rest_length" and n_angles
// lines "a1 a2 a3 rest_angle_radians".
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "Report.h"
using namespace ProtoMol::Report;
#include "CubicCellManager.h"
#include "ForceFactory.h"
#include "ForceGroup.h"
#include "GpuNonbondedForce.h"
#include "LeapfrogIntegrator.h"
#include "PeriodicBoundaryConditions.h"
#include "ScalarStructure.h"
#include "SystemForce.h"
#include "Topology.h"
#include "Vector3DBlock.h"
#include "Angle.h"
#include "Bond.h"
#include "blob_topology.h"
#include "topologyutilities.h"

using namespace ProtoMol;

int main(int argc, char** argv)
{
    if (argc < 8) {
        fprintf(stderr, "usage: gpu_leapfrog_driver <system.bin> <dynamics.bin> <out.bin> <steps> <dt> <gpu|cpu> "
                        "<definition>...\n");
        return 2;
    }
    Blob b;
    if (!read_blob(argv[1], b) || !b.periodic) { fprintf(stderr, "bad system file\n"); return 2; }
    const int steps = atoi(argv[4]);
    const double dt = atof(argv[5]);
    const bool gpu = strcmp(argv[6], "gpu") == 0;
    Topology<PeriodicBoundaryConditions, CubicCellManager>* topo = build_topology(b);
    std::vector<double> dyn(4 * (size_t)b.n);
    FILE* fd = fopen(argv[2], "rb");
    if (!fd || fread(dyn.data(), sizeof(double), dyn.size(), fd) != dyn.size()) { fprintf(stderr, "bad dynamics\n"); return 2; }
    fclose(fd);
    for (int i = 0; i < b.n; ++i) topo->atoms[i].scaledMass = dyn[i];
    for (size_t m = 0; m < topo->molecules.size(); ++m) {
        Real mass = 0.0;
        for (int a : topo->molecules[m].atoms) mass += topo->atoms[a].scaledMass;
        topo->molecules[m].mass = mass;
    }
    registerGpuForceExemplars();
    ForceGroup* group = new ForceGroup();
    for (int a = 7; a < argc; ++a) {
        std::string err;
        Force* f = ForceFactory::make(err, argv[a], std::vector<Value>());
        GpuNonbondedForce* g = dynamic_cast<GpuNonbondedForce*>(f);
        if (!g) { fprintf(stderr, "ForceFactory could not make '%s': %s\n", argv[a], err.c_str()); return 3; }
        if (gpu) {
            group->addSystemForce(g);
        } else {
            // the reference's own force of the same id and parameters, made by
            // its own make() from the values the factory parsed
            std::vector<Parameter> par;
            g->reference()->getParameters(par);
            std::vector<Value> vals;
            for (const Parameter& p : par) vals.push_back(p.value);
            Force* c = g->reference()->make(err, vals);
            SystemForce* cpu = dynamic_cast<SystemForce*>(c);
            if (!cpu) { fprintf(stderr, "reference force for '%s': %s\n", argv[a], err.c_str()); return 3; }
            group->addSystemForce(cpu);
        }
    }
    Vector3DBlock pos(b.n), vel(b.n);
    for (int i = 0; i < b.n; ++i) {
        pos[i] = Vector3D(b.pos[3 * i], b.pos[3 * i + 1], b.pos[3 * i + 2]);
        vel[i] = Vector3D(dyn[b.n + 3 * i], dyn[b.n + 3 * i + 1], dyn[b.n + 3 * i + 2]);
    }
    buildMolecularCenterOfMass(&pos, topo);
    buildMolecularMomentum(&vel, topo);
    ScalarStructure en;
    en.molecularVirial(false);
    en.virial(false);
    LeapfrogIntegrator* lf = new LeapfrogIntegrator(dt, group);
    const char* cons = getenv("LF_CONSTRAINTS");
    if (cons && *cons) {
        FILE* fc = fopen(cons, "r");
        int nb = 0, na = 0, shake_iter = 0, rattle_iter = 0;
        double shake_eps = 0.0, rattle_eps = 0.0;
        if (!fc || fscanf(fc, "%d %d %lf %d %lf %d", &nb, &na, &shake_eps, &shake_iter, &rattle_eps, &rattle_iter) != 6) {
            fprintf(stderr, "bad constraints file\n");
            return 2;
        }
        for (int k = 0; k < nb; ++k) {
            int a1, a2;
            double r;
            if (fscanf(fc, "%d %d %lf", &a1, &a2, &r) != 3) { fprintf(stderr, "bad bond\n"); return 2; }
            topo->bonds.push_back(Bond(a1, a2, 0.0, r));
            topo->atoms[a1].mybonds.push_back((int)topo->bonds.size() - 1);
            topo->atoms[a2].mybonds.push_back((int)topo->bonds.size() - 1);
        }
        for (int k = 0; k < na; ++k) {
            Angle ang;
            if (fscanf(fc, "%d %d %d %lf", &ang.atom1, &ang.atom2, &ang.atom3, &ang.restAngle) != 4) {
                fprintf(stderr, "bad angle\n");
                return 2;
            }
            topo->angles.push_back(ang);
        }
        fclose(fc);
        if (shake_eps > 0.0 && shake_iter > 0)
            lf->adoptPostDriftOrNextModifier(lf->createShakeModifier(shake_eps, shake_iter));
        if (rattle_eps > 0.0 && rattle_iter > 0)
            lf->adoptPostStepModifier(lf->createRattleModifier(rattle_eps, rattle_iter));
    }
    lf->initialize(topo, &pos, &vel, &en);
    lf->run(steps);
    const double epot = en.potentialEnergy();
    const double ekin = kineticEnergy(topo, &vel);
    FILE* out = fopen(argv[3], "wb");
    if (!out) return 4;
    double hdr[2] = {epot, ekin};
    fwrite(hdr, sizeof(double), 2, out);
    for (int i = 0; i < b.n; ++i) { double p3[3] = {pos[i].x, pos[i].y, pos[i].z}; fwrite(p3, sizeof(double), 3, out); }
    for (int i = 0; i < b.n; ++i) { double v3[3] = {vel[i].x, vel[i].y, vel[i].z}; fwrite(v3, sizeof(double), 3, out); }
    fclose(out);
    fprintf(stderr, "gpu evaluations: %lld\n", GpuNonbondedForce::evaluations());
    return 0;
}
