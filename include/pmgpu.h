/*
 * pmgpu.h -- C ABI of the B200 nonbonded force path (libpmgpu.so).
 *
 * The library evaluates ProtoMol's nonbonded system forces on one GPU:
 *   - the cell-list cutoff force NonbondedCutoffSystemForce with
 *     OneAtomPair / OneAtomPairTwo of LennardJones, Coulomb and
 *     CoulombEwaldReal under C1, C2, Cutoff and Shift switching
 *     (forces/NonbondedCutoffSystemForce.h:63-74, forces/OneAtomPair.h:127-188,
 *     forces/OneAtomPairTwo.h:131-199);
 *   - the particle-mesh Ewald force NonbondedPMEwaldSystemForce with
 *     -real / -reciprocal / -correction and B-spline interpolation
 *     (forces/NonbondedPMEwaldSystemForce.h:271-349).
 *
 * One pmgpu_system mirrors a ProtoMol Topology<PeriodicBoundaryConditions,
 * CubicCellManager> (atoms, exclusion table, Lennard-Jones table, box, cell
 * size).  One pmgpu_force mirrors one force object made by ForceFactory from
 * its keyword string.  pmgpu_evaluate mirrors SystemForce::evaluate
 * (forces/SystemForce.h:18-76) for one or several forces of a ForceGroup:
 * forces and energies are ACCUMULATED into the caller's arrays (+=), never
 * overwritten, exactly as the reference accumulates into its Vector3DBlock and
 * ScalarStructure.
 *
 * Plain C types only; every call returns a status code (PMGPU_OK = 0) and
 * pmgpu_last_error() returns the message of the last failure.  A context is
 * not thread-safe; it owns one CUDA stream.  There is no CPU fallback: without
 * a usable GPU every call that needs one fails with PMGPU_ERR_CUDA.
 */
#ifndef PMGPU_H
#define PMGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PMGPU_ABI_VERSION 1

/* status codes */
#define PMGPU_OK 0
#define PMGPU_ERR_ARG 1           /* invalid argument (reference: doMake errMsg / report << error) */
#define PMGPU_ERR_CUDA 2          /* CUDA runtime error or no device */
#define PMGPU_ERR_OVERFLOW 3      /* non-finite or out-of-range force (fixed-point range) */
#define PMGPU_ERR_STATE 4         /* call order: topology / box not set, size mismatch */
#define PMGPU_ERR_UNSUPPORTED 5   /* combination the reference does not register */
#define PMGPU_ERR_NOMEM 6         /* device allocation failed */
#define PMGPU_ERR_CAPACITY 7      /* a caller-provided capacity was too small */

/* ExclusionClass (topology/ExclusionTable.h) */
#define PMGPU_EXCL_NONE 0
#define PMGPU_EXCL_MODIFIED 1
#define PMGPU_EXCL_FULL 2

/* pair potentials */
#define PMGPU_POT_NONE 0
#define PMGPU_POT_LENNARD_JONES 1     /* forces/LennardJonesForce.h:37-74 */
#define PMGPU_POT_COULOMB 2           /* forces/CoulombForce.h:41-57 */
#define PMGPU_POT_EWALD_REAL 3        /* forces/CoulombEwaldRealForce.h:45-73 */
/* look-up-table potentials over base/LookUpTableBase.h (cubic Hermite in
 * r^2, 2^PRE points per octave from 2^-4 A^2 to the octave holding rc^2).
 * For these the term's sw is the TABULATED switching function and the pair
 * applies UniversalSwitchingFunction with the table's cutoff
 * (forces/oneAtomContraints.h:24-31); registered
 * (factories/registerForceExemplarsCutoff.cpp:47-48,58,69,86,101,132-134):
 *   LENNARD_JONES_TABLE + C2; COULOMB_TABLE + CUTOFF or SHIFT;
 *   EWALD_REAL_TABLE + CUTOFF;
 *   LENNARD_JONES (C1, C2, CUTOFF) + EWALD_REAL_TABLE;
 *   LENNARD_JONES_TABLE + EWALD_REAL_TABLE or COULOMB_TABLE (SHIFT). */
#define PMGPU_POT_LENNARD_JONES_TABLE 4   /* forces/LennardJonesTableForce.h:81-101, PRE 7 */
#define PMGPU_POT_COULOMB_TABLE 5         /* forces/CoulombTableForce.h:83-108, PRE 6 */
#define PMGPU_POT_EWALD_REAL_TABLE 6      /* forces/CoulombEwaldRealTableForce.h:85-107, PRE 6 */

/* switching functions */
#define PMGPU_SW_UNIVERSAL 0          /* topology/UniversalSwitchingFunction.h */
#define PMGPU_SW_CUTOFF 1             /* topology/CutoffSwitchingFunction.h:64-68 */
#define PMGPU_SW_C1 2                 /* topology/C1SwitchingFunction.h:64-75 */
#define PMGPU_SW_C2 3                 /* topology/C2SwitchingFunction.h:64-82 */
#define PMGPU_SW_SHIFT 4              /* topology/ShiftSwitchingFunction.h */

/* arithmetic of a force */
#define PMGPU_PRECISION_MIXED 0       /* FP32 pair/spread/FFT/gather, int64 fixed-point forces, FP64 sums */
#define PMGPU_PRECISION_FP64 1        /* plain FP64 kernels, reference operation order */

/* evaluate flags */
#define PMGPU_FLAG_VIRIAL 1u          /* ScalarStructure::virial() (base/ScalarStructure.h:135) */
/* ScalarStructure::molecularVirial() (base/ScalarStructure.h:119): the
 * energies pointer of pmgpu_evaluate then points to a pmgpu_energies_mol,
 * d_energies of pmgpu_evaluate_device to 20 doubles; the molecule positions
 * come from pmgpu_set_molecule_positions.  As in ProtoMol, pairs of atoms of
 * different molecules then add to the atomic virial even without
 * PMGPU_FLAG_VIRIAL (OneAtomPair.h:174-185), and the reciprocal term's
 * scalarSum tensor reaches the molecular virial only with it (Grid.h:341-387). */
#define PMGPU_FLAG_MOLECULAR_VIRIAL 2u

typedef struct pmgpu_system pmgpu_system;
typedef struct pmgpu_force pmgpu_force;

/* ScalarStructure slots this path writes (base/ScalarStructure.h:25-54):
 * LENNARDJONES, COULOMB and VIRIALXX..VIRIALZZ (row major). */
typedef struct {
    double lennard_jones;
    double coulomb;
    double virial[9];
} pmgpu_energies;

/* The same slots plus MOLVIRIALXX..MOLVIRIALZZ (row major). */
typedef struct {
    double lennard_jones;
    double coulomb;
    double virial[9];
    double molecular_virial[9];
} pmgpu_energies_mol;

/* One NonbondedCutoffSystemForce.  n_terms = 1: OneAtomPair<Periodic, sw[0],
 * pot[0]>; n_terms = 2: OneAtomPairTwo<Periodic, sw[0], pot[0], sw[1],
 * pot[1]> with pot[0] = LENNARD_JONES.  cutoff[k] is the switching
 * function's -cutoff, switchon[k] the C2 -switchon, alpha[k] the
 * CoulombEwaldReal -alpha; algorithm_cutoff is the NonbondedCutoff -cutoff
 * that sizes the neighbour-cell deltas
 * (forces/NonbondedCutoffForce.h:111-129). */
typedef struct {
    int n_terms;
    int pot[2];
    int sw[2];
    double switchon[2];
    double cutoff[2];
    double alpha[2];
    double algorithm_cutoff;
    int precision;
} pmgpu_cutoff_params;

/* NonbondedPMEwaldSystemForce<Periodic, Cubic, real, reciprocal, correction,
 * BSpline, CutoffSwitchingFunction>; parameters in getParameters() order
 * (forces/NonbondedPMEwaldSystemForce.h:1078-1090): -gridsize nx ny nz,
 * -cutoff, -order (default 4), -accuracy (default 1e-6), -alpha (default -1:
 * bisection of erfc(alpha Rc)/Rc = accuracy). */
typedef struct {
    int real;
    int reciprocal;
    int correction;
    int grid[3];
    int order;
    double cutoff;
    double accuracy;
    double alpha;
    int precision;
} pmgpu_pme_params;

/* ---- context ------------------------------------------------------------ */

/* Replaces: constructing Topology<PeriodicBoundaryConditions, CubicCellManager>
 * (topology/Topology.h:19-72). Selects the CUDA device and creates a stream. */
int pmgpu_system_create(int device, pmgpu_system** out);
/* Also destroys every force still alive on the system; do not call
 * pmgpu_force_destroy on those afterwards. */
int pmgpu_system_destroy(pmgpu_system* sys);

/* Replaces the GenericTopology members the nonbonded forces read
 * (topology/GenericTopology.h:129-144, filled by frontend/buildTopology.cpp):
 * atoms[i].scaledCharge / .type / .molecule, lennardJonesParameters (T*T
 * entries of {A, B, A14, B14}), exclusions.getTable() (pairs a1 < a2 with the
 * table class) and coulombScalingFactor.  excl_check_class (may be NULL) is
 * the class ExclusionTable::check() returns for each table pair; it differs
 * from the table class only when the same pair was added twice with different
 * classes (topology/ExclusionTable.cpp:122-141). */
int pmgpu_set_topology(pmgpu_system* sys, int n_atoms, const double* scaled_charge,
                       const int* type, const int* molecule, int n_types,
                       const double* lj_table, int n_excl, const int* excl_pairs,
                       const int* excl_class, const int* excl_check_class,
                       double coulomb_scaling_factor);

/* Replaces PeriodicBoundaryConditions::set (topology/PeriodicBoundaryConditions.cpp:40-77)
 * and CubicCellManager(cellsize) (topology/CubicCellManager.cpp:11-16).
 * Each vector has 3 doubles.  Orthogonal boxes only. */
int pmgpu_set_box(pmgpu_system* sys, const double* e1, const double* e2, const double* e3,
                  const double* origin, double cell_size);

/* ---- forces ------------------------------------------------------------- */

/* Replaces NonbondedCutoffForce::doMake (forces/NonbondedCutoffForce.h:119-123). */
int pmgpu_cutoff_create(pmgpu_system* sys, const pmgpu_cutoff_params* params, pmgpu_force** out);

/* The look-up table a table potential evaluates; host only, needs no GPU.
 * Replaces the LookUpTableBase constructor of LennardJonesTableForce /
 * CoulombTableForce / CoulombEwaldRealTableForce (base/LookUpTableBase.h:115-205)
 * for the tabulated switching function sw (switchon, cutoff) and alpha: per
 * entry 4 doubles per tabulated function (value, gradient, 2nd and 3rd
 * interpolation coefficient; LennardJonesTable: the A part, then the B part),
 * entries 2^PRE per octave of r^2 from 2^-4.  Writes at most cap doubles
 * (table may be NULL) and returns the table's length, or -1 for a potential
 * or switching function that is not a registered table. */
long long pmgpu_lookup_table(int pot, int sw, double switchon, double cutoff, double alpha,
                             double* table, long long cap);

/* Replaces NonbondedSimpleFullSystemForce<OneAtomPair[Two]<Vacuum...>> made by
 * the factory (forces/NonbondedSimpleFullSystemForce.h:165-182,
 * factories/registerForceExemplarsSimpleFull.cpp:88-152): every pair once,
 * plain differences (no periodic image), the same potentials and switches
 * (algorithm_cutoff unused).  Needs no box. */
int pmgpu_full_create(pmgpu_system* sys, const pmgpu_cutoff_params* params, pmgpu_force** out);

/* Replaces NonbondedPMEwaldSystemForce::doMake (forces/NonbondedPMEwaldSystemForce.h:1099-1139);
 * rejects the same parameter sets with PMGPU_ERR_ARG (order < 2 or odd,
 * grid < order, cutoff <= 0, accuracy <= 0).  Term sets that no exemplar
 * registers (factories/registerForceExemplarsFastElectrostatic.cpp:50-55):
 * none of real / reciprocal / correction, or real + reciprocal without
 * correction, return PMGPU_ERR_UNSUPPORTED, as do grid sizes with a prime
 * factor above 7 and orders above 12. */
int pmgpu_pme_create(pmgpu_system* sys, const pmgpu_pme_params* params, pmgpu_force** out);

int pmgpu_force_destroy(pmgpu_force* force);

/* Splitting parameter a PME force uses (after the bisection, if any). */
int pmgpu_pme_alpha(pmgpu_force* force, double* alpha);

/* ---- evaluation ----------------------------------------------------------- */

/* Replaces SystemForce::evaluate for each force in turn (ForceGroup::
 * evaluateSystemForces, forces/ForceGroup.cpp:43-96).  positions: 3N
 * doubles (host), forces_accum: 3N doubles (host, +=), energies (host, +=).
 * Blocks until the results are on the host. */
int pmgpu_evaluate(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces,
                   const double* positions, double* forces_accum,
                   pmgpu_energies* energies, unsigned flags);

/* Same with DEVICE pointers: d_positions (3N doubles), d_forces_accum (3N
 * doubles, +=), d_energies (11 doubles laid out as pmgpu_energies, +=).
 * Asynchronous on the system's stream; errors detected on the device are
 * reported by the next pmgpu_synchronize(). */
int pmgpu_evaluate_device(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces,
                          const double* d_positions, double* d_forces_accum,
                          double* d_energies, unsigned flags);

int pmgpu_synchronize(pmgpu_system* sys);

/* GenericTopology::molecules[m].position for m = 0 .. n_molecules - 1 (3
 * doubles each, host), the positions the molecular virial measures from
 * (OneAtomPair.h:178-179, NonbondedPMEwaldSystemForce.h:917-919); ProtoMol
 * sets them with buildMolecularCenterOfMass (topology/topologyutilities.cpp:
 * 761-769) or minimalImage.  n_molecules must be the topology's largest
 * molecule id plus one.  The copy is ordered on the system's stream before
 * the next evaluation.  The vacuum all-pairs force has no molecular virial
 * here (PMGPU_ERR_UNSUPPORTED), nor do the resident integrator runs. */
int pmgpu_set_molecule_positions(pmgpu_system* sys, int n_molecules, const double* positions);

/* The system's CUDA stream (a cudaStream_t). */
void* pmgpu_stream(pmgpu_system* sys);

/* Number of kernels the library launched since the system was created. */
long long pmgpu_launch_count(pmgpu_system* sys);

/* Profiling mode: while enabled, every evaluation records CUDA events around
 * its phases (and is not replayed from a CUDA graph).  Enabling resets the
 * accumulated times.  Replaces the reference's TimerStatistic / "force time"
 * wrappers (base/TimerStatistic.h:19-31, forces/SystemTimeForce.cpp). */
int pmgpu_set_profiling(pmgpu_system* sys, int enable);

/* Accumulated device milliseconds per phase since profiling was enabled:
 * ms[0] binning, [1] cutoff pair kernels, [2] PME correction, [3] PME
 * spread, [4] PME FFT + convolution, [5] PME gather, [6] finalize + energy
 * reduction, [7] cluster-pair list of the mixed cutoff kernel, [8] the
 * FP64 reciprocal energy transform of a mixed PME force; *evals =
 * number of profiled evaluations.  Synchronizes. */
int pmgpu_phase_times(pmgpu_system* sys, double* ms, int n, long long* evals);

/* Copies the last error message (NUL-terminated) into buf. */
int pmgpu_last_error(pmgpu_system* sys, char* buf, int len);

/* ---- differentiation (backward of pmgpu_evaluate) --------------------------
 * The reference has no adjoint; its analytic Hessian (integrators/
 * Hessian.cpp:456-623 with ReducedHessLennardJones.cpp:7-51,
 * ReducedHessCoulomb.cpp:8-43 and the switches' hessian(),
 * C2SwitchingFunction.cpp:45-53) is what the Hessian-vector product below
 * reproduces for the pair terms, for the NML integrators
 * (integrators/NormModeInt.cpp:368-415).  pmgpu_evaluate is the forward pass;
 * this backward pass recomputes the pair terms (nothing is stored) in the
 * forces' precision (FP64 or mixed) and ACCUMULATES (+=), host arrays:
 *   dE_dq   N:  dE/d(scaled charge) of all the forces (pair terms, PME
 *               reciprocal via the convolved potential, correction, self and
 *               charged-system terms);
 *   dE_dlj  T*T*4: dE/d(LJ table entry) in pmgpu_set_topology's layout
 *               {A, B, A14, B14}; each pair's derivative is split evenly
 *               between (t_i, t_j) and (t_j, t_i), so the gradient w.r.t. a
 *               symmetric entry t != t' is G[t][t'] + G[t'][t];
 *   hv      N*3: (H v), the Hessian of the energy applied to v (the
 *               negative force Jacobian-vector product): the pair terms, the
 *               PME reciprocal term (the charges' derivative along v spread
 *               on a second grid, the same convolution, then a gather of the
 *               B-splines' second derivatives on the potential and of their
 *               gradient on the convolved derivative) and the correction
 *               term's excluded-pair blocks (NonbondedPMEwaldSystemForce.h:
 *               942-981); PMEwald -real with lattice images is refused
 *               (PMGPU_ERR_UNSUPPORTED);
 *   energies 2: the pair terms' LJ and Coulomb energies (a check).
 * Any output may be NULL.  Table potentials differentiate their cubic
 * interpolant (exact inside an interval; C1 across intervals). */
int pmgpu_adjoint(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces, const double* positions,
                  const double* v, double* dE_dq, double* dE_dlj, double* hv, double* energies);

/* ---- batches of independent systems ---------------------------------------
 * The reference evaluates one system per process (ForceGroup::
 * evaluateSystemForces, forces/ForceGroup.cpp:70-82, once per replica or
 * per MPI rank).  A batch evaluates many independent systems of uneven size
 * with ONE CUDA graph launch: every member's forces run on that member's own
 * streams, all branching from the batch's stream, so small systems fill the
 * GPU together.  Members are (system, forces, device buffers) triples; the
 * results are those of pmgpu_evaluate_device on each member (accumulated,
 * +=).  The graph is captured on the first pmgpu_batch_evaluate and again
 * whenever a member's buffers, box, topology or forces change. */
typedef struct pmgpu_batch pmgpu_batch;
int pmgpu_batch_create(int device, pmgpu_batch** out);
int pmgpu_batch_destroy(pmgpu_batch* batch);
/* Adds a member: n_forces forces of sys evaluated on the device buffers
 * d_positions (N x 3), d_forces_accum (N x 3, +=), d_energies (11, +=). */
int pmgpu_batch_add(pmgpu_batch* batch, pmgpu_system* sys, int n_forces, pmgpu_force* const* forces,
                    const double* d_positions, double* d_forces_accum, double* d_energies, unsigned flags);
/* One graph launch of every member's evaluation, asynchronous on the batch's
 * stream (pmgpu_batch_stream). */
int pmgpu_batch_evaluate(pmgpu_batch* batch);
/* one_launch = 1 (the default): the members' column-path mixed cutoff
 * forces run their pair kernels as ONE persistent launch over every
 * member's (system, chunk) work items, between the members' own lists and
 * the rest of their evaluations (members must be distinct systems; up to
 * 1024); 0: each member's pair kernel on its own stream.  The results are
 * the same bit for bit; the next evaluation recaptures the graph. */
int pmgpu_batch_set_pair_launch(pmgpu_batch* batch, int one_launch);
/* Waits for the batch and reports the first member failure (for
 * PMGPU_ERR_CAPACITY, the member's list has been grown: evaluate again). */
int pmgpu_batch_synchronize(pmgpu_batch* batch);
int pmgpu_batch_last_error(pmgpu_batch* batch, char* buf, int len);
void* pmgpu_batch_stream(pmgpu_batch* batch);

/* ---- launch tuning -----------------------------------------------------
 * No counterpart in the reference (its CPU loops have nothing to tune).  The
 * launch shapes of a system's evaluation: the cluster-pair list's work
 * chunks, the mixed pair kernel's resident blocks, the PME FFT's lines per
 * block, whether PME runs on a second stream beside the pair kernels, and
 * whether mixed cutoff forces take the FP64 pair kernels.  Results do not
 * depend on the first four beyond the last bits of the fixed-point grouping
 * (a chunk's partial sums are rounded together); fp64_pairs gives the FP64
 * kernels' results, which hold every mixed-precision bound.  Defaults: 16, 0
 * (the occupancy limit), 16, 1, 0. */
typedef struct pmgpu_tuning {
    int chunk_entries;        /* cluster-list entries per chunk of pair work: 4..64 */
    int pair_blocks_per_sm;   /* resident blocks of the mixed pair kernel per SM: 0 (occupancy limit) or 1..8 */
    int fft_lines;            /* lines per block of the strided PME FFT passes, at most: 1..16 (z passes: twice) */
    int pme_concurrent;       /* 1: PME on a second stream beside the pair kernels; 0: after them */
    int fp64_pairs;           /* 1: mixed cutoff forces run the FP64 pair kernels (no cluster list, no
                                 near-pair pass: the shorter launch chain, faster on a few hundred atoms) */
    double ms_per_eval;       /* pmgpu_autotune: the measured time of the chosen tuning */
} pmgpu_tuning;
int pmgpu_get_tuning(pmgpu_system* sys, pmgpu_tuning* out);
/* PMGPU_ERR_ARG for a value out of range; the next evaluation is recaptured. */
int pmgpu_set_tuning(pmgpu_system* sys, const pmgpu_tuning* tuning);
/* Project-written autotuner: times candidate tunings on these forces and
 * these positions (host, N x 3), evals evaluations each after two warm-up
 * ones, with CUDA events on the system's stream; a coordinate search over
 * the five parameters, two sweeps (fp64_pairs only on systems of at most
 * 4,096 atoms; pmgpu_batch_autotune leaves it at 0).  Keeps the fastest for the system's later
 * evaluations and returns it (with its time) in *best.  Synchronous; uses
 * the system's own scratch buffers (no caller output is touched). */
int pmgpu_autotune(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces, const double* positions,
                   unsigned flags, int evals, pmgpu_tuning* best);
/* The same search for a batch: each candidate is applied to every member and
 * timed as whole batch launches.  The members' output buffers receive the
 * timed evaluations (zero them before the next real one). */
int pmgpu_batch_autotune(pmgpu_batch* batch, int evals, pmgpu_tuning* best);

/* ---- dense Hessian ----------------------------------------------------------
 * Hessian::evaluate's LJ / Coulomb pair blocks (integrators/Hessian.cpp:
 * 456-623; ReducedHessLennardJones.cpp:7-51, ReducedHessCoulomb.cpp:8-43,
 * switches C2SwitchingFunction::hessian C2SwitchingFunction.cpp:45-53) of the
 * pair terms of cutoff, all-pairs and PME-real forces: the 3N x 3N second
 * derivative of their energy at the host positions, row-major, added (+=)
 * to hessian.  The matrix the normal-mode integrators diagonalise
 * (NormalModeUtilities).  Up to 8,192 atoms (PMGPU_ERR_CAPACITY);
 * PMGPU_ERR_UNSUPPORTED for the PME reciprocal and correction terms. */
int pmgpu_hessian(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces, const double* positions,
                  double* hessian);

/* ---- integration ---------------------------------------------------------
 * LeapfrogIntegrator::run(n_steps) (integrators/LeapfrogIntegrator.cpp:
 * 107-120; doHalfKickdoDrift :47-68, doKickdoDrift :70-101, doHalfKick
 * StandardIntegrator.cpp:83-96), with the SHAKE and RATTLE modifiers of
 * pmgpu_set_constraints when they are set, on device buffers that
 * stay in HBM: per step one kick/drift kernel and one evaluation of the
 * forces (the captured graph), with no host round trip.  d_forces must hold
 * the forces at d_positions on entry (the integrator's forces after
 * initialize(), or after the previous run); on return d_positions and
 * d_velocities are advanced by n_steps * timestep (fs), d_forces and
 * d_energies (11, cleared per evaluation like calculateForces) belong to the
 * final positions.  d_mass: N atom masses (amu, atoms[i].scaledMass).
 * Asynchronous on the system's stream; failures of the evaluations
 * (PMGPU_ERR_CAPACITY: a list outgrew its size, grown for the next run)
 * surface at pmgpu_synchronize, and the run is then to be repeated from its
 * starting state. */
int pmgpu_leapfrog_run(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces, const double* d_mass,
                       double* d_positions, double* d_velocities, double* d_forces, double* d_energies,
                       double timestep, int n_steps, unsigned flags);

/* Bond constraints of pmgpu_leapfrog_run: SHAKE after every drift
 * (ModifierShake, integrators/ModifierShake.cpp:21-99, a post-drift
 * modifier) and RATTLE after every step (ModifierRattle,
 * ModifierRattle.cpp:19-80, a post-step modifier), as protomol.cpp:553-577
 * attaches them for shake / rattle in a .conf; an epsilon <= 0 or a
 * max_iter <= 0 leaves that modifier out.  atoms: 2 per constraint, with
 * rest_length, in the order buildRattleShakeBondConstraintList gives them
 * (topology/topologyutilities.cpp:782-860: every bond, then the H-H pair of
 * every angle between two light atoms).  Each sweep updates the
 * constraints in that order within every group of constraints that share
 * atoms (the reference's sequential sweep); the mean error over all
 * constraints (ModifierMetaShake / ModifierMetaRattle::calcError) decides
 * the next sweep.  SHAKE's bond vectors start as the positions a run
 * starts from; RATTLE's virial term enters d_energies with
 * PMGPU_FLAG_VIRIAL.  One CTA runs the sweeps (sized for molecules of small
 * systems).  n_constraints = 0 removes them; a pmgpu_set_topology with
 * another atom count does too.  Masses are the run's d_mass. */
int pmgpu_set_constraints(pmgpu_system* sys, int n_constraints, const int* atoms, const double* rest_length,
                          double shake_epsilon, int shake_max_iter, double rattle_epsilon, int rattle_max_iter);

/* Sweeps of SHAKE or RATTLE that stopped at their max_iter since the
 * constraints were first set (the reference reports each with a warning,
 * ModifierShake.cpp:85-91).  Synchronizes; -1 on a CUDA error. */
long long pmgpu_constraint_limit_hits(pmgpu_system* sys);

/* ImpulseIntegrator::run(n_steps) (integrators/ImpulseIntegrator.cpp,
 * MTSIntegrator.cpp, StandardIntegrator.cpp:24-35) over an inner Leapfrog of
 * `timestep` fs, without modifiers: per outer step a half kick with the slow
 * forces (outer timestep = cyclelength * timestep), pmgpu_leapfrog_run of
 * cyclelength steps with the fast forces, the slow forces at the new
 * positions, a half kick.  On entry d_slow_forces / d_fast_forces hold the
 * two groups' forces at d_positions; on return all of positions,
 * velocities, forces and the two energy arrays (11 each) belong to the final
 * positions (the reference adds both levels into one ScalarStructure: their
 * sum).  Asynchronous on the system's stream, like pmgpu_leapfrog_run. */
int pmgpu_impulse_run(pmgpu_system* sys, int n_slow, pmgpu_force* const* slow, int n_fast, pmgpu_force* const* fast,
                      const double* d_mass, double* d_positions, double* d_velocities, double* d_slow_forces,
                      double* d_fast_forces, double* d_slow_energies, double* d_fast_energies, double timestep,
                      int cyclelength, int n_steps, unsigned flags);

/* ---- diagnostics (parity tests) ----------------------------------------- */

/* Cell of every atom from the GPU binning of the last evaluation, as
 * buildCellLists computes it (topology/buildCellLists.cpp:11-38): 3N ints
 * (x, y, z) and the grid dims. */
int pmgpu_get_cells(pmgpu_system* sys, int* cells, int* dims);

/* No counterpart in the reference (diagnostic).  The cluster layout the
 * mixed-precision cutoff forces of the last evaluation ran on:
 * PMGPU_LAYOUT_COLUMNS (fixed-point coordinates in z-sorted columns, boxes
 * well above twice the cutoff), PMGPU_LAYOUT_CELLS (clusters inside the
 * reference cells: smaller boxes, the small-grid mode, or a system whose
 * columns or clusters exceeded the column layout's limits),
 * PMGPU_LAYOUT_FP64 (the FP64 pair kernels, tuning fp64_pairs), or 0 (none
 * yet). */
#define PMGPU_LAYOUT_CELLS 1
#define PMGPU_LAYOUT_COLUMNS 2
#define PMGPU_LAYOUT_FP64 3
int pmgpu_pair_layout(pmgpu_system* sys);

/* No counterpart in the reference, whose cutoff force rebuilds its cell lists
 * at every evaluation (forces/NonbondedCutoffSystemForce.h:63-74).  A reused
 * pair list for the column layout: the list is built with the cutoff plus
 * `skin` (A) and kept for `rebuild_every` evaluations of the same forces, the
 * positions refreshed each time; the within-cutoff decision stays exact per
 * evaluation, so the interacting pair set is the reference's as long as no
 * atom moves more than skin / 2 between rebuilds.  One that does makes the
 * evaluation report PMGPU_ERR_CAPACITY and the list is rebuilt at the next
 * (pmgpu_evaluate repeats the evaluation by itself).  Applies to force groups
 * with one mixed-precision cutoff force on the column layout; rebuild_every =
 * 1 (the default) rebuilds at every evaluation.  pmgpu_pair_list_builds
 * counts the lists built so far. */
int pmgpu_set_pair_list(pmgpu_system* sys, double skin, int rebuild_every);
long long pmgpu_pair_list_builds(pmgpu_system* sys);

/* Evaluates one cutoff force (or a PME force with -real) in pair-recording
 * mode and returns the within-cutoff pair set: every (min, max) atom index
 * pair the force interacted, in no particular order.  *count receives the
 * number of pairs; PMGPU_ERR_CAPACITY if it exceeds cap. */
int pmgpu_get_pairs(pmgpu_system* sys, pmgpu_force* force, const double* positions,
                    long long* count, int* pairs, long long cap);

/* ---- allocation-free PME reciprocal term --------------------------------- */

/* No counterpart in the reference.  The PME reciprocal-space term (spread,
 * FFT with the convolution, gather; the mixed-precision kernels of a PME
 * force made with -reciprocal only) for callers that must not allocate GPU
 * memory: code whose device memory is owned by another allocator (a
 * framework's caching allocator or a memory pool sized to the whole GPU,
 * where a cudaMalloc fails or breaks the pool's accounting), or code that
 * may not call cudaMalloc / cudaFree at the point where the force is needed.
 * Nothing is allocated: the charge grid, spectrum, fixed-point forces and
 * energy records live in about 8.4 MB of statically reserved memory that
 * every GPU loading this library holds until the process exits.
 *   d_positions        N x 3 FP64 (absolute coordinates, orthogonal box),
 *   d_scaled_charges   N FP64 (charge * sqrt(332.0636), as the topology's),
 *   box                the three edge lengths, grid the K per axis,
 *   order              even, 2..12; alpha > 0 (the Ewald splitting);
 *   d_forces_accum     N x 3 FP64, the forces are added (+=);
 *   d_energies         11 FP64: [1] += reciprocal energy and, with
 *                      PMGPU_FLAG_VIRIAL, [2..10] += virial (xx xy xz yx ...).
 * All pointers d_* are device memory on `device`.  Limits: N <= 65,536
 * atoms, Kx*Ky*Kz <= 262,144 (64^3), each K <= 1,024, Kx*Ky*(Kz/2+1) <=
 * 196,608 and Ky*(Kz/2+1) <= 8,192; larger sizes return PMGPU_ERR_CAPACITY.
 * Each K has prime factors 2, 3, 5 and 7 only, as for pmgpu_pme_create;
 * other grid sizes return PMGPU_ERR_UNSUPPORTED before any launch.
 * Runs on `stream` (NULL: the legacy default stream) and returns when the
 * results are written; PMGPU_ERR_OVERFLOW for non-finite forces.  The first
 * call on a device looks up the scratch address and initialises it (and
 * synchronizes the device), so it should come before any stream capture.
 * Every call shares the one scratch area: calls that overlap on the GPU
 * (from several host threads) race and must be serialised by the caller. */
int pmgpu_pme_reciprocal_static(int device, int n_atoms, const double* d_positions,
                                const double* d_scaled_charges, const double box[3], const int grid[3],
                                int order, double alpha, double* d_forces_accum, double* d_energies,
                                unsigned flags, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PMGPU_H */
