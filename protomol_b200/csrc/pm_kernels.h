// pm_kernels.h -- host-side launchers of the libpmgpu kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pm_internal.cuh"

namespace pm {

// ---------------------------------------------------------------- binning
struct BinArgs {
    int n;
    const double* pos;          // 3N raw positions
    const double* q;            // N scaled charges
    const int* type;
    const int* mol;
    Pbc pbc;
    CellGrid grid;
    int* cell_lin;              // N
    int* cell3;                 // 3N
    int* counts;                // ncell (zeroed by the launcher)
    int* fill;                  // ncell (zeroed by the launcher)
    int* start;                 // ncell + 1
    int* tmp;                   // N
    int* sorted;                // N: original index per sorted slot
    int* slot_of;               // N: sorted slot per original index
    float4* spos;               // N
    int4* smeta;                // N
    double4* spos64;            // N (raw FP64 position + charge) or null
    int* status;
};
// Cell binning by counting sort (K1): buildCellLists' cell of every atom in
// exact FP64, CSR cell offsets, stable (ascending index) order within a cell.
int launch_bin(const BinArgs& a, cudaStream_t s, long long* launches);

// ---------------------------------------------------------------- pair force
struct TermF {
    int pot, sw;
    float cut2, on2, s1, s2, s3;          // C2
    float c1_15_1, c1_05_3, c1_15_3;      // C1
    float sh_a, sh_b;                      // Shift
    float alpha, two_alpha_pi;             // EwaldReal
};

struct TermD {
    int pot, sw;
    double cut2, on2, s1, s2, s3;
    double c1_15_1, c1_05_3, c1_15_3;
    double sh_a, sh_b;
    double alpha, two_alpha_pi;
};

struct PairArgs {
    // cell-sorted system
    const int* start;
    const float4* spos;
    const int4* smeta;
    const double4* spos64;
    const double* pos;           // raw positions, original order (exact rechecks)
    // exclusions (check() classes), window masks + CSR for larger deltas
    const uint32_t* xfull;
    const uint32_t* xmod;
    const int* xrow;             // N + 1
    const int2* xent;            // (partner, class) for deltas > window
    // LJ table
    const float4* ljf;
    const double4* ljd;
    int n_types;
    // enumeration
    const int4* deltas;          // nd neighbour-cell deltas (reference order)
    const float4* doff;          // FP32 offset delta * real cell size
    int nd;
    CellGrid grid;
    Pbc pbc;
    int wrap;                    // per-pair minimal image in FP32 (small grids)
    float lx, ly, lz, ilx, ily, ilz;
    // physics
    int n_terms;
    TermF tf[2];
    TermD td[2];
    float cut2f;                 // pair test (largest switching cutoff^2)
    double cut2d;
    float guard;                 // relative guard band of the FP32 tests
    float csf;
    double csfd;
    int virial;
    // outputs
    unsigned long long* facc;    // 3 per sorted slot
    double scale;
    double* erec;                // energy records, one per block
    int* status;
    int* rec_pairs;              // pair recording (diagnostic) or null
    unsigned long long* rec_count;
    long long rec_cap;
};

// Combination id of the registered OneAtomPair[Two] templates.
int pair_combo_id(int n_terms, const int* pot, const int* sw);
int launch_pair_mixed(const PairArgs& a, int combo, int blocks, cudaStream_t s, long long* launches);
int launch_pair_fp64(const PairArgs& a, int combo, int blocks, cudaStream_t s, long long* launches);
int pair_blocks(const CellGrid& g, int nd);

// ---------------------------------------------------------------- PME
struct PmeArgs {
    int n;
    const double* pos;           // raw positions (original order)
    const double* q;
    const int* sorted;           // cell-sorted order of atoms (locality) or null
    const int* slot_of;          // original -> sorted slot (force accumulation)
    int kx, ky, kz, kzh, order;
    double hxr, hyr, hzr;        // K/L
    int offx, offy, offz;        // -(P-1)/2 + K
    long long* qgrid;            // int64 fixed-point charge grid K^3
    void* cgrid;                 // complex half spectrum kx*ky*kzh (float2 or double2)
    void* rgrid;                 // real grid K^3 (float or double)
    const void* tw;              // twiddle tables, concatenated for x, y, z (float2/double2)
    int twx, twy, twz;           // offsets into tw
    const double* bfac;          // per axis: modX[kx], modY[ky], modZ[kz] (concatenated)
    const double* efac;          // per axis: expX, expY, expZ
    double piVr;                 // 1 / (pi V)
    double fac;                  // pi^2 / alpha^2
    double wr, lr, hr;           // 1/Lx, 1/Ly, 1/Lz
    unsigned long long* facc;
    double scale;
    double qscale;               // fixed-point scale of the charge grid
    double* erec;
    int* status;
    int virial;
};
int launch_pme_reciprocal(const PmeArgs& a, int fp64, cudaStream_t s, long long* launches,
                          double* erec_base, int* erec_used);

struct CorrArgs {
    int n_excl;
    const int2* pairs;
    const int* cls;
    const double* pos;
    const double* q;
    const int* slot_of;
    Pbc pbc;
    double alpha, alpha2, two_alpha_pi, csf;
    unsigned long long* facc;
    double scale;
    double* erec;
    int* status;
    int virial;
};
int launch_pme_correction(const CorrArgs& a, cudaStream_t s, long long* launches, int* blocks_used);

// ---------------------------------------------------------------- finalize
int launch_finalize(int n, const unsigned long long* facc, const int* sorted, double inv_scale,
                    double* fout, cudaStream_t s, long long* launches);
int launch_energy_reduce(const double* erec, int nrec, double* out, cudaStream_t s, long long* launches);

}  // namespace pm
