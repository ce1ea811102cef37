/*
 * pmoracle.h -- CPU restatement of ProtoMol's nonbonded force path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity checker for the GPU kernels
 * in protomol_b200/csrc; nothing in the product links or calls it.  Only the
 * tests, the smoke check and the benchmark's CPU-baseline leg may load it.
 *
 * Every function restates a reference function and cites it (paths relative
 * to the ProtoMol source tree).  The arithmetic is plain IEEE double in the
 * reference's operation order, compiled with -ffp-contract=off, so that on the
 * same inputs it reproduces the compiled reference bit for bit (checked by
 * tests/test_oracle_vs_reference.py against oracle/_ref).
 */
#ifndef PMORACLE_H
#define PMORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ExclusionClass (topology/ExclusionTable.h) */
enum { PMO_EXCL_NONE = 0, PMO_EXCL_MODIFIED = 1, PMO_EXCL_FULL = 2 };

/* pair potentials (forces/LennardJonesForce.h, CoulombForce.h,
 * CoulombEwaldRealForce.h) */
enum { PMO_POT_NONE = 0, PMO_POT_LJ = 1, PMO_POT_COULOMB = 2, PMO_POT_EWALD_REAL = 3,
       /* look-up-table potentials (forces/LennardJonesTableForce.h,
        * CoulombTableForce.h, CoulombEwaldRealTableForce.h over
        * base/LookUpTableBase.h): sw is the tabulated switching function,
        * the pair itself is Universal with the table's cutoff */
       PMO_POT_LJ_TABLE = 4, PMO_POT_COULOMB_TABLE = 5, PMO_POT_EWALD_REAL_TABLE = 6 };

/* switching functions (topology/C1SwitchingFunction.h, C2..., Cutoff...,
 * Shift...); UNIVERSAL = no
 * switching and no cutoff test */
enum { PMO_SW_UNIVERSAL = 0, PMO_SW_CUTOFF = 1, PMO_SW_C1 = 2, PMO_SW_C2 = 3, PMO_SW_SHIFT = 4 };

typedef struct {
    int n_atoms;
    const double* pos;          /* 3N, x y z */
    const double* q;            /* N scaled charges */
    const int* type;            /* N */
    const int* mol;             /* N */
    int n_types;
    const double* lj;           /* T*T*4: A, B, A14, B14 */
    int n_excl;
    const int* excl;            /* 3E: a1, a2, table class */
    const int* excl_check;      /* E: class returned by check(); NULL = same */
    double box[12];             /* e1, e2, e3, origin */
    double csf;                 /* coulombScalingFactor */
    double cell_size;           /* CubicCellManager cellsize */
    /* GenericTopology::molecules[m].position, 3 per molecule: with it the
     * molecular virial is computed (ScalarStructure::molecularVirial());
     * NULL: off */
    const double* mol_pos;
    int no_virial;              /* ScalarStructure::virial() false */
} pmo_system;

/* One NonbondedCutoffSystemForce: OneAtomPair (n_terms = 1) or
 * OneAtomPairTwo (n_terms = 2). */
typedef struct {
    int n_terms;
    int pot[2];
    int sw[2];
    double switchon[2];         /* C2 only */
    double sw_cutoff[2];
    double alpha[2];            /* EwaldReal only */
    double algo_cutoff;         /* NonbondedCutoff -cutoff (cell deltas) */
} pmo_cutoff_params;

/* NonbondedPMEwaldSystemForce<Periodic, Cubic, real, reciprocal, correction,
 * BSpline, Cutoff> */
typedef struct {
    int real, reciprocal, correction;
    int grid[3];
    int order;
    double cutoff;
    double accuracy;
    double alpha;               /* <= 0: bisection default */
} pmo_pme_params;

typedef struct {
    double lennard_jones;
    double coulomb;
    double virial[9];
    long long n_pairs;          /* interactions computed (pair set size) */
    double alpha;               /* PME: splitting parameter used */
    double e_real, e_recip, e_intra, e_self, e_charged;   /* PME parts */
    int out_of_grid;            /* atoms whose cell fell outside the grid */
    double mol_virial[9];       /* MOLVIRIALXX..MOLVIRIALZZ (row major) */
} pmo_result;

/* buildMolecularCenterOfMass (topology/topologyutilities.cpp:761-769): the
 * centre of mass of every molecule (atoms in index order, Kahan-summed as
 * molecularCenterOfMass, :729-759), 3 per molecule into centers; mass NULL
 * = unit masses.  Returns the number of molecules (max molecule id + 1). */
int pmo_molecular_centers(const pmo_system* s, const double* mass, double* centers);

/* ModifierShake::doExecute (integrators/ModifierShake.cpp:21-99) with
 * ModifierMetaShake::calcError (ModifierMetaShake.cpp): sweeps over the K
 * constraints in list order until the mean error is at most eps or max_iter
 * sweeps are exceeded; pos, vel updated, last (the previous SHAKE's
 * positions) set to pos at the end.  dt = timestep / TIMEFACTOR.  Returns
 * the number of sweeps (max_iter + 1 when the limit was hit). */
int pmo_shake(int n_cons, const int* atoms, const double* rest, const double* mass, int n_atoms,
              double* pos, double* vel, double* last, double dt, double eps, int max_iter);

/* ModifierRattle::doExecute (integrators/ModifierRattle.cpp:19-80) with
 * ModifierMetaRattle::calcError; virial (9, +=) or NULL. */
int pmo_rattle(int n_cons, const int* atoms, const double* rest, const double* mass,
               const double* pos, double* vel, double dt, double eps, int max_iter, double* virial);

/* Cell of every atom as buildCellLists computes it, and the grid dims.
 * cells: 3N ints. Returns 0. */
int pmo_cell_assign(const pmo_system* s, int* cells, int* dims);

/* Cutoff force: forces += (3N), result accumulates energies/virial.
 * pairs (optional, capacity cap pairs) receives the (min, max) index pair of
 * every interaction evaluated, in enumeration order. */
int pmo_cutoff_force(const pmo_system* s, const pmo_cutoff_params* p,
                     double* forces, pmo_result* r,
                     int* pairs, long long cap);

/* PME force: forces += (3N). */
int pmo_pme_force(const pmo_system* s, const pmo_pme_params* p,
                  double* forces, pmo_result* r);

/* All-pairs force with vacuum boundary conditions
 * (NonbondedSimpleFullSystemForce<OneAtomPair[Two]<Vacuum, ...>>). */
int pmo_simple_full_force(const pmo_system* s, const pmo_cutoff_params* p,
                          double* forces, pmo_result* r);

/* Dense 3N x 3N Hessian of the pair terms (integrators/Hessian.cpp:456-623),
 * vacuum (plain differences) or periodic (minimal image); H +=.  Returns -1
 * for terms without a Hessian block there. */
int pmo_pair_hessian(const pmo_system* s, const pmo_cutoff_params* p, int vacuum, double* H);

/* One LookUpTableBase of a table potential over r^2 in [2^floor(log2 0.1),
 * the octave holding rc^2]: values per entry (4 per tabulated function: value,
 * gradient, 2nd and 3rd interpolation coefficients); entries = 2 for
 * LennardJonesTable (A and B parts), 1 otherwise.  Returns the number of
 * doubles written to table (at most cap), -1 for a bad term. */
long long pmo_lookup_table(int pot, int sw, double switchon, double cutoff, double alpha,
                           double* table, long long cap);

/* The poly5 erfc approximation (base/mathutilities.cpp:29-40). */
double pmo_poly5(double ar);

/* Unnormalised 3-D complex FFT on an nx*ny*nz row-major array of
 * (re, im) pairs; sign -1 or +1.  Exposed for tests. */
int pmo_fft3d(double* data, int nx, int ny, int nz, int sign);

#ifdef __cplusplus
}
#endif
#endif
