// blob_topology.h -- the system file of protomol_b200.systems.System.save
// and the reference Topology<PeriodicBoundaryConditions, CubicCellManager>
// built from it with the GenericTopology members buildTopology fills
// (frontend/buildTopology.cpp): atoms, molecules, Lennard-Jones table,
// exclusions.  Shared by the drop-in drivers.
#ifndef BLOB_TOPOLOGY_H
#define BLOB_TOPOLOGY_H
#include <cstdio>
#include <cstring>
#include <vector>

#include "CubicCellManager.h"
#include "ExclusionType.h"
#include "PeriodicBoundaryConditions.h"
#include "Topology.h"

namespace ProtoMol
{
struct Blob {
    int n, t, e, periodic;
    double box[12], csf, cell;
    std::vector<double> pos, q, lj;
    std::vector<int> type, mol, excl, check;
};

inline bool read_blob(const char* path, Blob& b)
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


inline Topology<PeriodicBoundaryConditions, CubicCellManager>* build_topology(const Blob& b)
{
    Vector3D e1(b.box[0], b.box[1], b.box[2]), e2(b.box[3], b.box[4], b.box[5]),
        e3(b.box[6], b.box[7], b.box[8]), o(b.box[9], b.box[10], b.box[11]);
    Topology<PeriodicBoundaryConditions, CubicCellManager>* tp = new Topology<PeriodicBoundaryConditions, CubicCellManager>(
        b.csf, ExclusionType(ExclusionType::ONE4MODIFIED), PeriodicBoundaryConditions(e1, e2, e3, o),
        CubicCellManager(b.cell));
    // the GenericTopology members buildTopology fills (frontend/buildTopology.cpp)
    tp->atoms.resize(b.n);
    int nmol = 0;
    for (int i = 0; i < b.n; ++i) {
        tp->atoms[i].type = b.type[i];
        tp->atoms[i].scaledCharge = b.q[i];
        tp->atoms[i].scaledMass = 1.0;
        tp->atoms[i].molecule = b.mol[i];
        if (b.mol[i] + 1 > nmol) nmol = b.mol[i] + 1;
    }
    tp->molecules.resize(nmol);
    for (int i = 0; i < b.n; ++i) tp->molecules[b.mol[i]].atoms.push_back(i);
    tp->lennardJonesParameters.resize(b.t);
    for (int i = 0; i < b.t; ++i)
        for (int j = 0; j < b.t; ++j) {
            const double* p = &b.lj[4 * ((size_t)i * b.t + j)];
            LennardJonesParameters par;
            par.A = p[0]; par.B = p[1]; par.A14 = p[2]; par.B14 = p[3];
            tp->lennardJonesParameters.set(i, j, par);
        }
    tp->exclusions.resize(b.n);
    for (int k = 0; k < b.e; ++k)
        tp->exclusions.add(b.excl[3 * k], b.excl[3 * k + 1], (ExclusionClass)b.excl[3 * k + 2]);
    for (int k = 0; k < b.e; ++k)
        if (b.check[k] != b.excl[3 * k + 2])
            tp->exclusions.add(b.excl[3 * k], b.excl[3 * k + 1], (ExclusionClass)b.check[k]);
    tp->exclusions.optimize();

    return tp;
}
}  // namespace ProtoMol
#endif
