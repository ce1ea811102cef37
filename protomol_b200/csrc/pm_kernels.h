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
    int* counts;                // ncell; zero on entry, and again on exit
    int* done;                  // blocks of k_bin_count finished (zero on entry)
    int* start;                 // ncell + 1
    int* tmp;                   // N
    int* sorted;                // N: original index per sorted slot
    int* slot_of;               // N: sorted slot per original index
    float4* spos;               // N: FP32 (hi) cell-relative x, y, z and charge
    float4* slo;                // N: FP32 remainders (lo) of the same four values
    int4* smeta;                // N
    double4* spos64;            // N (raw FP64 position + charge) or null
    int* skey;                  // N: Morton key of the cell-relative position
    int* cstart;                // ncell + 1: first cluster of each cell
    int* ccell;                 // cluster -> cell
    float4* cbox;               // 2 per cluster: bounding box lo, hi
    int ncl_cap;                // capacity of ccell / cbox
    int* status;
};
constexpr int kCluster = 8;     // atoms per cluster (z-sorted slab of a cell)
// Cell binning by counting sort (K1): buildCellLists' cell of every atom in
// exact FP64, CSR cell offsets, stable (ascending index) order within a cell.
int launch_bin(const BinArgs& a, cudaStream_t s, long long* launches);

// ---------------------------------------------------------------- column clusters
// The mixed pair path of boxes well above twice the cutoff: atoms in
// unsigned 32-bit fixed point of the box (x / L * 2^32, so that the int32
// difference of two atoms is their minimal-image displacement exactly), in
// columns of an x-y grid (~4 A side) sorted by z; every run of 8 atoms of a
// column is an i-cluster, each half of it a 4-atom j-cluster.
constexpr int kColAtoms = 1024;  // atoms a column may hold (more: the cell-cluster path)
struct ColGrid {
    int ncx, ncy, ncol;
    int rx, ry;                  // column reach of the list
    double lx, ly, lz;           // box edges
    double mnx, mny, mnz;        // box minimum corner (origin - L / 2)
    float sx, sy;                // column side
    float lxf, lyf, lzf;         // box edges (FP32)
    float sch[3], scl[3];        // L / 2^32 per axis, FP32 hi + lo
    float zext;                  // largest z extent of an i-cluster that keeps every tile's image unique
};

// z index of a column's j-clusters: kZBins bins of L_z / kZBins; per column
// and bin edge b (0 .. kZBins) the first j-cluster whose box ends at or above
// b L_z / kZBins, then the first whose box starts above it
constexpr int kZBins = 64;
constexpr int kZIndex = 2 * (kZBins + 1);   // ints per column

struct ColBinArgs {
    int n;
    const double* pos;
    const double* q;
    const int* type;
    const int* mol;
    Pbc pbc;
    CellGrid grid;               // reference cells (bit-exact assignment, reported)
    int* cell3;                  // 3N reference cell of every atom
    ColGrid g;
    unsigned* qfix;              // 3N fixed-point position (atom order)
    int* col;                    // N column of every atom
    int* counts;                 // ncol; zero on entry, and again on exit
    int* done;                   // blocks of the count kernel finished (zero on entry)
    int* colstart;               // ncol + 1: first atom of each column (compact order)
    int* ccstart;                // ncol + 1: first i-cluster of each column
    int* tmp;                    // N
    int4* cq;                    // slot: qx, qy, qz, charge (FP32 hi, as bits)
    int4* cm;                    // slot: original index (-1: padding), type, molecule, charge (FP32 lo, as bits)
    int* slot_of;                // N: slot of every atom
    float4* ibox;                // 2 per i-cluster: lo, hi (A, box frame [0, L))
    float4* jbox;                // 2 per j-cluster
    int* ccol;                   // i-cluster -> column
    int4* corg;                  // i-cluster -> fixed-point position of its first atom (virial origin)
    int* zidx;                   // kZIndex per column: the z index of its j-clusters
    int ncl_cap;                 // i-cluster capacity
    int* status;
};
// K0: up to kZeroRanges ranges of 4-byte words set to zero in one launch
constexpr int kZeroRanges = 10;
struct ZeroRanges {
    unsigned* p[kZeroRanges];
    long long words[kZeroRanges];
    int count;
};
int launch_zero(const ZeroRanges& z, cudaStream_t s, long long* launches);
// K1c: fixed point, columns, z order, clusters and their boxes
int launch_col_bin(const ColBinArgs& a, cudaStream_t s, long long* launches);
// K1r: between rebuilds of a reused pair list, the current fixed-point
// positions into the slots (and the reference cells); an atom farther than
// half the skin from where the list was built sets kStatusListStale
int launch_col_refresh(const ColBinArgs& a, double half_skin, cudaStream_t s, long long* launches);

// ---------------------------------------------------------------- pair force
// FP32 constants of one term; the *_lo members are the FP32 remainders of
// constants that multiply every pair (their rounding would otherwise bias
// the energy sum the same way for all pairs)
struct TermF {
    int pot, sw;
    float cut2, on2, s1, s2, s3;          // C2
    float s1_lo, s3_lo;
    float c1_15_1, c1_05_3, c1_15_3;      // C1
    float c1_15_1_lo, c1_05_3_lo, c1_15_3_lo;
    float sh_a, sh_b;                      // Shift
    float sh_a_lo, sh_b_lo;
    float alpha, two_alpha_pi;             // EwaldReal
    float alpha_lo, two_alpha_pi_lo;
    // table potentials: the FP32 copy of the look-up table (tab_step floats
    // per entry), hashed on the top bits of the FP32 r^2 (tab_shift = 23 -
    // PRE); tab_first and tab_last are float offsets
    const float* tab;
    int tab_step, tab_first, tab_last, tab_shift;
};

struct TermD {
    int pot, sw;
    double cut2, on2, s1, s2, s3;
    double c1_15_1, c1_05_3, c1_15_3;
    double sh_a, sh_b;
    double alpha, two_alpha_pi;
    // table potentials: LookUpTableBase's FP64 table, hashed on the top
    // bits of the FP64 r^2 (tab_shift = 52 - PRE); double offsets
    const double* tab;
    int tab_step, tab_last, tab_shift;
    long long tab_first;
};

struct PairArgs {
    // cell-sorted system
    const int* start;
    const int* cstart;           // first 8-atom cluster of each cell
    const int* ccell;            // cluster -> cell
    const float4* cbox;          // cluster bounding boxes (lo, hi)
    int ncl_cap;                 // bound on the number of clusters
    const float4* spos;
    const float4* slo;
    const int4* smeta;
    const double4* spos64;
    const double* pos;           // raw positions, original order (exact rechecks)
    // exclusions (check() classes), window masks + CSR for larger deltas
    const uint32_t* xfull;
    const uint32_t* xmod;
    const int* xrow;             // N + 1
    const int2* xent;            // (partner, class) for deltas > window
    // LJ table: FP32 hi/lo pairs {A_hi, B_hi, A_lo, B_lo} for normal pairs
    // (ljn) and for 1-4 modified pairs (ljm); FP64 {A, B, A14, B14} (ljd)
    const float4* ljn;
    const float4* ljm;
    const double4* ljd;
    int n_types;
    // enumeration
    const int4* deltas;          // nd neighbour-cell deltas (reference order)
    const float4* doff;          // FP32 offset delta * real cell size
    int nd;
    // the mixed kernel's half shell: the positive half of the deltas (each
    // unordered cell pair once, every cell the same work), or in the
    // small-grid mode the reference's deltas with the B > A rule
    const int4* hdeltas;
    const float4* hoff;          // FP32 hi offsets
    const float4* hoff_lo;       // FP32 remainders of the offsets
    int nh;
    int half_rule;               // 1: skip B < A (small-grid mode)
    CellGrid grid;
    Pbc pbc;
    int wrap;                    // per-pair minimal image in FP32 (small grids)
    float lx, ly, lz, ilx, ily, ilz;
    float lx_lo, ly_lo, lz_lo;   // FP32 remainders of the box lengths
    // physics
    int n_terms;
    TermF tf[2];
    TermD td[2];
    float cut2f;                 // pair test (largest switching cutoff^2)
    double cut2d;
    float guard;                 // relative guard band of the FP32 tests
    float near2;                 // mixed kernel: pairs with FP32 r^2 below this get FP64 energies (0: none)
    int2* near;                  // those pairs: sorted slots i, j | 1 << 30 for a 1-4 (modified) pair
    int* near_count;
    int* near_need;
    int near_cap;
    float csf;
    double csfd;
    int virial;
    // outputs
    unsigned long long* facc;    // 3 per sorted slot
    double scale;
    double* erec;                // energy records (component-major, see kERec)
    int erec_stride;
    int* status;
    int* rec_pairs;              // pair recording (diagnostic) or null
    unsigned long long* rec_count;
    long long rec_cap;
    // mixed kernel: cluster-pair list, chunks of work, fixed-point sums
    int2* plist;                 // {first j slot, (delta + 1) | nj << 16 | i-cluster mask << 24}
    int plist_cap;
    int4* chunks;                // {first i slot, i atoms (<= 32), first entry, entries}
    int chunk_cap;
    int* plist_count;            // entries written (zeroed before the list kernel)
    int* plist_need;             // entries needed when a capacity was exceeded
    int* chunk_count;
    int* chunk_need;
    int* chunk_next;             // work counter of the pair kernel
    const double4* hoff64;       // FP64 half-shell offsets (hi + lo), virial
    unsigned long long* efix;    // 11 int64 sums (scale 2^32): LJ, Coulomb, virial
    int blocks_per_sm;           // resident blocks of the mixed pair kernel per SM (0: the occupancy limit)
    int chunk;                   // cluster-list entries per chunk of pair work
    // column-cluster path (K2a' / K2b'): slot data, cluster boxes, grid
    const int4* cq;
    const int4* cm;
    const float4* ibox;
    const float4* jbox;
    const int* zidx;             // kZIndex per column (ColBinArgs::zidx)
    const int* ccstart;          // ncol + 1
    const int* ccol;
    const int4* corg;            // virial origin of every i-cluster
    int4* clist;                 // column-path entries (the plist buffer): {jc | flags << 25, o.x, o.y, o.z};
                                 // o = O_c(j) - O_c(i) + t L (FP32 bits), the tile's virial offset
    int icl_cap;                 // i-clusters the list kernel's grid covers
    ColGrid cg;
    const double* qorig;         // charges, types in atom order (FP64 near-pair energies)
    const int* torig;
    float list_skin;             // the column list includes pairs up to the cutoff plus this (reused lists)
    // molecular virial (launch_pair_molvir): molecule positions, records
    const double* molpos;        // 3 per molecule
    double* mrec;
    int mrec_stride;
};

// Combination id of the registered OneAtomPair[Two] templates.
int pair_combo_id(int n_terms, const int* pot, const int* sw);
// K2a: the cluster-pair list; K2b: the mixed kernel over it
int launch_cluster_list(const PairArgs& a, cudaStream_t s, long long* launches);
int launch_pair_mixed(const PairArgs& a, int combo, cudaStream_t s, long long* launches);
// K2c: FP64 energies of the near pairs listed by the mixed pair kernel
int launch_near_energy(const PairArgs& a, int combo, int n_atoms, cudaStream_t s, long long* launches);
// K2a' / K2b' / K2c': the column-cluster list, pair kernel and near-pair energies
int launch_col_list(const PairArgs& a, cudaStream_t s, long long* launches);
int launch_pair_col(const PairArgs& a, int combo, cudaStream_t s, long long* launches);
// K11: the column-path pair kernels of up to kBatchPairMax systems (a
// batch's members, the same combination of terms) as one persistent launch
constexpr int kBatchPairMax = 1024;
struct BatchPairArgs {
    const PairArgs* args;        // device copy of every member's pair arguments
    int n;
    int* next;                   // work counter (zero before the launch)
};
int launch_pair_col_batch(const BatchPairArgs& b, int combo, cudaStream_t s, long long* launches);
int launch_near_energy_col(const PairArgs& a, int combo, int n_atoms, cudaStream_t s, long long* launches);
long long col_list_estimate(int n_atoms, const ColGrid& g, double volume, double cutoff);
long long col_chunk_estimate(long long entries, int n_atoms, const ColGrid& g, int chunk);
int launch_pair_fp64(const PairArgs& a, int combo, int blocks, cudaStream_t s, long long* launches);
// the molecular virial records (kMRec) of a cutoff force over the cell-sorted
// order, one per block (blocks as launch_pair_fp64), no forces or energies
int launch_pair_molvir(const PairArgs& a, int combo, int blocks, cudaStream_t s, long long* launches);
int pair_blocks(const CellGrid& g, int nd);
// blocks of the mixed kernel (4 warps, one energy record per warp)
// estimated cluster-pair list entries and chunks of a system
long long plist_estimate(int n_atoms, const CellGrid& g, int nh);
long long chunk_estimate(int n_atoms, const CellGrid& g, int nh, int chunk);

// ---------------------------------------------------------------- adjoint
// K10: gradients of the pair energy w.r.t. charges and the LJ table, and the
// Hessian-vector product, recomputed pair by pair (all ordered pairs, exact
// FP64 minimal image and cutoff decision; math in FP64 or FP32)
struct AdjArgs {
    int n;
    const double* pos;           // 3N, original order
    const double* q;             // N scaled charges
    const int* type;
    const int* mol;
    Pbc pbc;
    int periodic;                // 0: vacuum (plain differences)
    const uint32_t* xfull;
    const uint32_t* xmod;
    const int* xrow;
    const int2* xent;
    const double4* ljd;          // T x T of {A, B, A14, B14}
    int n_types;
    int n_terms;
    TermD td[2];
    int modify;                  // the switches are applied (one of them modifies)
    int use_cut;                 // pair test r^2 <= cut2d (0: all pairs)
    double cut2d;
    double csf;
    const double* v;             // 3N displacement for H v, or null
    double* dq;                  // N (+=) or null
    double* dlj;                 // T x T x 4 (+=) or null
    double* hv;                  // 3N (+=) or null
    double* hess;                // 3N x 3N row-major (+=) or null: the dense pair Hessian
    double* energy;              // 2 (+=): LJ, Coulomb, or null
    // forward mode (the vacuum all-pairs force): forces in atom order
    // (fixed point) and one energy/virial record per block
    unsigned long long* facc;    // 3N or null
    double scale;
    int* status;
    double* erec;                // records or null
    int erec_stride;
    int virial;
};
int launch_pair_adjoint(const AdjArgs& a, int fp64, cudaStream_t s, long long* launches);
// the same backward pass for a cutoff force over the cell list (the cell
// pairs and pair set of launch_pair_fp64; p holds the cell-sorted order):
// dq, dlj, hv and energy of a (facc, hess and erec are not written)
int launch_pair_adjoint_cells(const PairArgs& p, const AdjArgs& a, int fp64, int blocks, cudaStream_t s,
                              long long* launches);
// records (blocks) of one launch_pair_adjoint
int adjoint_blocks(int n);

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
    int erec_stride;
    int* status;
    int virial;
    int fft_lines;               // lines per CTA of the strided FFT passes, at most (0: 16)
    int energy64_apart;          // mixed: the FP64 energy transform is its own stage (kStageEnergy64)
    // mixed precision: the reciprocal energy and virial from an FP64 forward
    // transform of the charge grid (double2 half spectrum, FP64 twiddles),
    // launched after the gather; null: from the FP32 convolution pass
    void* cgrid64;
    const void* tw64;
    // kStageMolvir: the molecular virial records (kMRec) of the reciprocal
    // forces against each atom's offset from its molecule's position
    const int* mol;
    const double* molpos;        // 3 per molecule
    Pbc pbc;
    double* mrec;
    int mrec_stride;
    // Hessian-vector product (kStageSpreadDir, kStageHvpGather): the
    // displacement v (3N, atom order), the output H v (3N, +=) and the
    // convolved grid of the directional-derivative charges
    const double* dir;
    double* hv;
    const void* rgrid_d;
};
constexpr int kStageSpread = 0, kStageFft = 1, kStageGather = 2;
constexpr int kStagePotential = 3;   // dE/dq~ = phi at the atoms, into (double*)facc
constexpr int kStageEnergy64 = 4;    // mixed: the FP64 energy transform alone (energy64_apart)
constexpr int kStageMolvir = 5;      // the reciprocal forces' molecular virial (after the gather)
constexpr int kStageSpreadDir = 6;   // H v: the charges' derivative along v spread into qgrid
constexpr int kStageHvpGather = 7;   // H v: second-derivative gather on rgrid plus gradient gather on rgrid_d
// molecular virial records one kStageMolvir launch writes
int pme_molvir_blocks(int n);
// One stage of the reciprocal term: K3 spread, the five FFT passes with the
// fused convolution (K4/K5, writes energy records), or K6 gather.
int launch_pme_reciprocal(const PmeArgs& a, int fp64, cudaStream_t s, long long* launches,
                          double* erec_base, int* erec_used, int stage);
void pme_init_attributes();

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
    int erec_stride;
    int* status;
    int virial;
    double const_energy;         // point self + charged-system energy (added once)
    double const_virial;         // charged-system term on the virial diagonal
};
int launch_pme_correction(const CorrArgs& a, cudaStream_t s, long long* launches, int* blocks_used);

// realTerm with lattice images (boxes with an edge <= 2 rc): every unordered
// pair and every atom with itself, over the lattice vectors of
// PeriodicBoundaryConditions::buildLatticeVectors, in FP64
struct RealLatArgs {
    int n;
    const double* pos;
    const double* q;
    const int* mol;
    const uint32_t* xfull;
    const uint32_t* xmod;
    const int* xrow;
    const int2* xent;
    Pbc pbc;
    const double4* lattice;      // (0, 0, 0) first, then sorted by norm
    int n_lattice;
    double rc2, alpha, two_alpha_pi, csf;
    unsigned long long* facc;    // atom order
    double scale;
    double* erec;
    int erec_stride;
    int* status;
    int virial;
    const double* molpos;        // molecular virial mode (launch_pme_real_lattice_molvir)
    double* mrec;
    int mrec_stride;
};
int launch_pme_real_lattice(const RealLatArgs& a, cudaStream_t s, long long* launches, int* blocks_used);
// the lattice real space's molecular virial records (kMRec), no forces
int launch_pme_real_lattice_molvir(const RealLatArgs& a, cudaStream_t s, long long* launches, int* blocks_used);
int launch_pme_correction_adjoint(const CorrArgs& a, double* dq, cudaStream_t s, long long* launches);
// H v of the correction term's excluded pairs (3N, atom order, +=)
int launch_pme_correction_hvp(const CorrArgs& a, const double* v, double* hv, cudaStream_t s, long long* launches);

// ---------------------------------------------------------------- finalize
// forces of the three fixed-point accumulators (any may be null) added into
// fout in the caller's order; with pair_virial, the per-atom term
// sum p (x) F of the mixed pair forces (f32) as one FP64 record per block
struct FinArgs {
    int n;
    const unsigned long long* f32;      // mixed pair forces (whole-cell shifts), 2^32
    const unsigned long long* f32p;     // other mixed forces (PME, per-pair minimal image), 2^32
    const unsigned long long* f40;      // FP64 forces, 2^40
    const unsigned long long* a32;      // in atom order (PME): mixed, 2^32
    const unsigned long long* a40;      // in atom order (PME): FP64, 2^40
    const int* sorted;
    const float4* spos;
    const float4* slo;
    int pair_virial;
    // column-cluster pair forces (2^32) per slot, gathered through slot_of;
    // their virial from the fixed-point positions (cq) times L / 2^32
    const unsigned long long* c32;
    const int* c_slot_of;
    int c_slots;                         // slots of c32 / cq (an out-of-range slot_of adds nothing)
    const int4* cq;
    const int4* corg;                    // virial origin of each i-cluster (slot / 8)
    double cscale[3];
    double* fout;
    double* erec;
    int erec_stride;
};
int launch_finalize(const FinArgs& a, cudaStream_t s, long long* launches, int* records);
// sums the FP64 records and adds the int64 fixed-point sums (efix, scale 2^32)
int launch_energy_reduce(const double* erec, int stride, int nrec, const unsigned long long* efix,
                         double* out, cudaStream_t s, long long* launches);
// the molecular virial into out[11..19]: the records (kMRec) plus the virial
// slots of the reciprocal energy records in the given ranges (scalarSum's
// tensor, which ProtoMol adds to both virials); without the atomic virial
// (virial = 0) the records' inter-molecular atomic virial into out[2..10]
struct MolvirFinish {
    const double* mrec;
    int mstride, nmrec;
    const double* erec;
    int estride;
    int range_first[4], range_count[4];
    int nranges;
    int virial;
    double* out;
};
int launch_molvir_finish(const MolvirFinish& f, cudaStream_t s, long long* launches);

// Leapfrog kick / drift (LeapfrogIntegrator.cpp): the first step's half kick
// and drift, a middle step's kick and drift, the last half kick
// (kLeapfrogLast is also the lone half kick before and after RATTLE; the
// drift alone follows the second half kick)
constexpr int kLeapfrogFirst = 0, kLeapfrogMiddle = 1, kLeapfrogLast = 2, kLeapfrogDrift = 3;
int launch_leapfrog(int n, const double* mass, double* pos, double* vel, const double* force, double h, double hk,
                    int mode, cudaStream_t s, long long* launches);

// Bond constraints of the resident Leapfrog: SHAKE after every drift
// (ModifierShake, integrators/ModifierShake.cpp:21-99) and RATTLE after every
// step (ModifierRattle, ModifierRattle.cpp:19-80).  The constraints come
// grouped in clusters (connected through shared atoms), each cluster's
// constraints in the caller's list order; one thread sweeps a cluster
// sequentially, as the reference's Gauss-Seidel sweep treats it, and the
// mean error over all constraints (ModifierMetaShake::calcError,
// ModifierMetaRattle::calcError) decides the next sweep.  One CTA.
struct ConsArgs {
    int n_cons, n_clusters;
    const int* cl_start;         // n_clusters + 1
    const int2* atoms;           // per constraint, cluster order
    const double* rest;          // rest lengths
    const double* mass;
    double* pos;
    double* vel;
    const double* last;          // SHAKE: positions after the previous SHAKE
    double dt;                   // getTimestep() / Constant::TIMEFACTOR
    double eps;
    int max_iter;
    double* virial;              // RATTLE: 9 doubles (+=) or null
    int* hits;                   // sweeps that ended at max_iter (+1 each)
};
int launch_shake(const ConsArgs& a, cudaStream_t s, long long* launches);
int launch_rattle(const ConsArgs& a, cudaStream_t s, long long* launches);

}  // namespace pm
