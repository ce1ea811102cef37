// GpuNonbondedForce.cpp -- see GpuNonbondedForce.h.
#include "Report.h"
using namespace ProtoMol::Report;

#include "GpuNonbondedForce.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>

#include "BSpline.h"
#include "C1SwitchingFunction.h"
#include "C2SwitchingFunction.h"
#include "CellListEnumerator_periodicBoundaries.h"
#include "CoulombEwaldRealForce.h"
#include "CoulombEwaldRealTableForce.h"
#include "CoulombForce.h"
#include "CoulombTableForce.h"
#include "CubicCellManager.h"
#include "CutoffSwitchingFunction.h"
#include "ForceFactory.h"
#include "LennardJonesForce.h"
#include "LennardJonesTableForce.h"
#include "NonbondedCutoffSystemForce.h"
#include "NonbondedPMEwaldSystemForce.h"
#include "OneAtomPair.h"
#include "OneAtomPairTwo.h"
#include "PeriodicBoundaryConditions.h"
#include "ScalarStructure.h"
#include "ShiftSwitchingFunction.h"
#include "Topology.h"
#include "UniversalSwitchingFunction.h"
#include "Vector3DBlock.h"

namespace ProtoMol
{
	typedef PeriodicBoundaryConditions PBC;
	typedef Topology<PBC, CubicCellManager> PTopo;

	static_assert(sizeof(Vector3D) == 3 * sizeof(double), "Vector3DBlock must be packed x, y, z doubles");

	// One pmgpu_system per topology (shared by the GPU forces of a ForceGroup).
	struct GpuContext
	{
		pmgpu_system* sys = nullptr;
		size_t n = 0;
		double box[12];
		double cell = 0.0;
		bool dirty = true;            // upload the topology
		bool recheck = false;         // uncache(): upload it again only if it changed
		unsigned long long digest = 0;
	};

	// A digest of the topology members the GPU forces read, so that uncache()
	// (which the integrators call for box changes, Integrator.cpp:153) does
	// not re-upload an unchanged topology
	static unsigned long long topology_digest(const GenericTopology* topo)
	{
		unsigned long long h = 1469598103934665603ull;
		auto mix = [&h](const void* p, size_t n) {
			const unsigned char* c = (const unsigned char*)p;
			for (size_t k = 0; k < n; ++k) { h ^= c[k]; h *= 1099511628211ull; }
		};
		for (size_t i = 0; i < topo->atoms.size(); ++i) {
			mix(&topo->atoms[i].scaledCharge, sizeof(Real));
			mix(&topo->atoms[i].type, sizeof(topo->atoms[i].type));
			mix(&topo->atoms[i].molecule, sizeof(topo->atoms[i].molecule));
		}
		const std::vector<ExclusionPair>& tab = topo->exclusions.getTable();
		for (size_t k = 0; k < tab.size(); ++k) {
			mix(&tab[k].a1, sizeof(tab[k].a1)); mix(&tab[k].a2, sizeof(tab[k].a2)); mix(&tab[k].excl, sizeof(tab[k].excl));
		}
		int t = topo->lennardJonesParameters.size();
		for (int a = 0; a < t; ++a)
			for (int b = 0; b < t; ++b) {
				const LennardJonesParameters& p = topo->lennardJonesParameters(a, b);
				mix(&p.A, sizeof(p.A)); mix(&p.B, sizeof(p.B)); mix(&p.A14, sizeof(p.A14)); mix(&p.B14, sizeof(p.B14));
			}
		mix(&topo->coulombScalingFactor, sizeof(topo->coulombScalingFactor));
		return h;
	}

	static std::map<const GenericTopology*, GpuContext>& contexts()
	{
		static std::map<const GenericTopology*, GpuContext>* m = new std::map<const GenericTopology*, GpuContext>();
		return *m;
	}

	static void gpu_fail(pmgpu_system* sys, const std::string& what)
	{
		char buf[512] = {0};
		pmgpu_last_error(sys, buf, sizeof(buf));
		report << error << "[GpuNonbondedForce] " << what << ": " << buf << endr;
	}

	// Uploads the GenericTopology members the nonbonded forces read
	// (topology/GenericTopology.h:129-144) and the periodic box / cell size.
	static GpuContext& context_for(const GenericTopology* topo)
	{
		GpuContext& c = contexts()[topo];
		const PTopo* pt = dynamic_cast<const PTopo*>(topo);
		if (!pt)
			report << error << "[GpuNonbondedForce] needs Topology<PeriodicBoundaryConditions, CubicCellManager>" << endr;
		if (!c.sys) {
			const char* dev = getenv("PMGPU_DEVICE");
			if (pmgpu_system_create(dev ? atoi(dev) : 0, &c.sys) != PMGPU_OK)
				report << error << "[GpuNonbondedForce] no usable CUDA device" << endr;
		}
		double box[12];
		const Vector3D* v[4] = {&pt->boundaryConditions.e1(), &pt->boundaryConditions.e2(),
		                        &pt->boundaryConditions.e3(), &pt->boundaryConditions.origin()};
		for (int k = 0; k < 4; ++k) { box[3 * k] = v[k]->x; box[3 * k + 1] = v[k]->y; box[3 * k + 2] = v[k]->z; }
		double cell = pt->cellManager.getCellSize();
		if (c.recheck && !c.dirty && c.n == topo->atoms.size()) {
			c.dirty = topology_digest(topo) != c.digest;
			c.recheck = false;
		}
		if (c.dirty || c.n != topo->atoms.size()) {
			size_t n = topo->atoms.size();
			std::vector<double> q(n);
			std::vector<int> type(n), mol(n);
			for (size_t i = 0; i < n; ++i) {
				q[i] = topo->atoms[i].scaledCharge;
				type[i] = topo->atoms[i].type;
				mol[i] = topo->atoms[i].molecule;
			}
			int t = topo->lennardJonesParameters.size();
			std::vector<double> lj(4 * (size_t)t * t);
			for (int a = 0; a < t; ++a)
				for (int b = 0; b < t; ++b) {
					const LennardJonesParameters& p = topo->lennardJonesParameters(a, b);
					double* o = &lj[4 * ((size_t)a * t + b)];
					o[0] = p.A; o[1] = p.B; o[2] = p.A14; o[3] = p.B14;
				}
			const std::vector<ExclusionPair>& tab = topo->exclusions.getTable();
			std::vector<int> pairs(2 * tab.size()), cls(tab.size()), chk(tab.size());
			for (size_t k = 0; k < tab.size(); ++k) {
				pairs[2 * k] = tab[k].a1; pairs[2 * k + 1] = tab[k].a2;
				cls[k] = (int)tab[k].excl;
				chk[k] = (int)topo->exclusions.check(tab[k].a1, tab[k].a2);
			}
			if (pmgpu_set_topology(c.sys, (int)n, q.data(), type.data(), mol.data(), t, lj.data(), (int)tab.size(),
			                       pairs.data(), cls.data(), chk.data(), topo->coulombScalingFactor) != PMGPU_OK)
				gpu_fail(c.sys, "set_topology");
			c.n = n;
			c.cell = -1.0;
			c.dirty = false;
			c.recheck = false;
			c.digest = topology_digest(topo);
		}
		if (c.cell != cell || memcmp(c.box, box, sizeof(box)) != 0) {
			if (pmgpu_set_box(c.sys, box, box + 3, box + 6, box + 9, cell) != PMGPU_OK) gpu_fail(c.sys, "set_box");
			memcpy(c.box, box, sizeof(box));
			c.cell = cell;
		}
		return c;
	}

	// ForceGroup::evaluateSystemForces (forces/ForceGroup.cpp:43-96) calls the
	// system forces of a group one after another into the same forces and
	// energies.  The GPU forces of a group run as ONE pmgpu_evaluate (one
	// upload of the positions, one download of the forces; PME beside the
	// pair kernels): the first round of calls evaluates each force alone and
	// records the order in which the group's GPU forces come; from the next
	// round on, the first of them evaluates the whole group and the others
	// find their share done.  A group that changes its GPU forces between
	// rounds is an error (PMGPU_COALESCE=0 evaluates every force alone).
	struct GroupRun
	{
		std::vector<GpuNonbondedForce*> seq;
		bool learned = false;
		size_t next = 0;
	};

	// never destroyed: the factory's exemplars are deleted at exit, after
	// function-local statics constructed later than the factory
	static std::map<std::pair<const void*, const void*>, GroupRun>& group_runs()
	{
		static std::map<std::pair<const void*, const void*>, GroupRun>* m =
			new std::map<std::pair<const void*, const void*>, GroupRun>();
		return *m;
	}

	// host staging of the molecule positions (never destroyed, as above)
	static std::vector<double>& molecule_positions()
	{
		static std::vector<double>* v = new std::vector<double>();
		return *v;
	}

	static long long g_evaluations = 0;
	long long GpuNonbondedForce::evaluations() { return g_evaluations; }

	static bool coalescing()
	{
		const char* c = getenv("PMGPU_COALESCE");
		return !(c && strcmp(c, "0") == 0);
	}

	GpuNonbondedForce::GpuNonbondedForce(SystemForce* reference, int kind, int n_terms, const int* pot,
	                                     const int* sw, int precision)
		: SystemForce(), myReference(reference), myKind(kind), myTerms(n_terms), myPrecision(precision),
		  myForce(nullptr), mySystem(nullptr)
	{
		for (int k = 0; k < 2; ++k) {
			myPot[k] = (pot && k < n_terms) ? pot[k] : 0;
			mySw[k] = (sw && k < n_terms) ? sw[k] : 0;
		}
	}

	GpuNonbondedForce::~GpuNonbondedForce()
	{
		if (myForce && mySystem) pmgpu_force_destroy(myForce);
		delete myReference;
		// a group with this force is learned again
		for (auto it = group_runs().begin(); it != group_runs().end();)
			if (std::find(it->second.seq.begin(), it->second.seq.end(), this) != it->second.seq.end())
				it = group_runs().erase(it);
			else
				++it;
	}

	int GpuNonbondedForce::defaultPrecision()
	{
		const char* p = getenv("PMGPU_PRECISION");
		return (p && strcmp(p, "fp64") == 0) ? PMGPU_PRECISION_FP64 : PMGPU_PRECISION_MIXED;
	}

	std::string GpuNonbondedForce::getKeyword() const { return myReference->getKeyword(); }
	std::string GpuNonbondedForce::getIdNoAlias() const { return myReference->getIdNoAlias(); }
	void GpuNonbondedForce::getParameters(std::vector<Parameter>& p) const { myReference->getParameters(p); }
	unsigned int GpuNonbondedForce::getParameterSize() const { return myReference->getParameterSize(); }

	void GpuNonbondedForce::uncache()
	{
		myReference->uncache();
		// the box is compared at every evaluation; the topology is compared
		// with its digest at the next one
		for (auto& kv : contexts()) kv.second.recheck = true;
	}

	Force* GpuNonbondedForce::doMake(std::string& errMsg, std::vector<Value> values) const
	{
		// the reference validates and stores the parameters
		Force* made = myReference->make(errMsg, values);
		if (!made) return NULL;
		SystemForce* ref = dynamic_cast<SystemForce*>(made);
		return new GpuNonbondedForce(ref, myKind, myTerms, myPot, mySw, defaultPrecision());
	}

	static double real_of(const Parameter& p)
	{
		Real r = 0.0;
		p.value.get(r);
		return r;
	}

	bool GpuNonbondedForce::ensureForce(const GenericTopology* topo)
	{
		GpuContext& c = context_for(topo);
		if (myForce && mySystem == c.sys) return true;
		std::vector<Parameter> par;
		myReference->getParameters(par);
		int r;
		if (myKind == 0) {
			// OneAtomPair[Two]::getParameters order: force1, switch1, force2,
			// switch2, then the algorithm -cutoff (NonbondedCutoffForce.h:111-117)
			pmgpu_cutoff_params cp;
			memset(&cp, 0, sizeof(cp));
			cp.n_terms = myTerms;
			size_t k = 0;
			for (int t = 0; t < myTerms; ++t) {
				cp.pot[t] = myPot[t];
				cp.sw[t] = mySw[t];
				// a table potential's parameters are its tabulated switching
				// function's, then -alpha (CoulombEwaldRealTableForce.h:126-131);
				// the pair's Universal switch has none
				const bool table = myPot[t] >= PMGPU_POT_LENNARD_JONES_TABLE;
				if (myPot[t] == PMGPU_POT_EWALD_REAL) cp.alpha[t] = real_of(par[k++]);
				if (mySw[t] == PMGPU_SW_C2) { cp.switchon[t] = real_of(par[k++]); cp.cutoff[t] = real_of(par[k++]); }
				else if (mySw[t] != PMGPU_SW_UNIVERSAL) cp.cutoff[t] = real_of(par[k++]);
				if (table && myPot[t] == PMGPU_POT_EWALD_REAL_TABLE) cp.alpha[t] = real_of(par[k++]);
			}
			cp.algorithm_cutoff = real_of(par[k]);
			cp.precision = myPrecision;
			r = pmgpu_cutoff_create(c.sys, &cp, &myForce);
		} else {
			// NonbondedPMEwaldSystemForce::getParameters (:1078-1090)
			pmgpu_pme_params pp;
			memset(&pp, 0, sizeof(pp));
			std::string id = myReference->getIdNoAlias();
			pp.real = id.find(" -real") != std::string::npos;
			pp.reciprocal = id.find(" -reciprocal") != std::string::npos;
			pp.correction = id.find(" -correction") != std::string::npos;
			int g[3];
			for (int a = 0; a < 3; ++a) { par[a].value.get(g[a]); pp.grid[a] = g[a]; }
			pp.cutoff = real_of(par[3]);
			int order = 4;
			par[4].value.get(order);
			pp.order = order;
			pp.accuracy = real_of(par[5]);
			pp.alpha = real_of(par[6]);
			pp.precision = myPrecision;
			r = pmgpu_pme_create(c.sys, &pp, &myForce);
		}
		if (r != PMGPU_OK) gpu_fail(c.sys, "force creation");
		mySystem = c.sys;
		return true;
	}

	void GpuNonbondedForce::evaluate(const GenericTopology* topo, const Vector3DBlock* positions,
	                                 Vector3DBlock* forces, ScalarStructure* energies)
	{
		ensureForce(topo);
		if (positions->size() == 0) return;
		std::vector<pmgpu_force*> run(1, myForce);
		if (coalescing()) {
			GroupRun& g = group_runs()[std::make_pair((const void*)forces, (const void*)energies)];
			if (!g.learned) {
				if (!g.seq.empty() && g.seq[0] == this) {
					g.learned = true;                // the group's order repeats: learned
					g.next = 0;
				} else {
					if (std::find(g.seq.begin(), g.seq.end(), this) != g.seq.end())
						report << error << "[GpuNonbondedForce] a GPU force evaluated twice in one force group" << endr;
					g.seq.push_back(this);           // still learning: this force alone
				}
			}
			if (g.learned) {
				if (g.seq[g.next] != this)
					report << error << "[GpuNonbondedForce] the GPU forces of a force group changed between steps "
					       << "(set PMGPU_COALESCE=0 to evaluate each force alone)" << endr;
				const bool first = g.next == 0;
				g.next = (g.next + 1) % g.seq.size();
				if (!first) return;                  // included in the group's evaluation
				run.clear();
				for (GpuNonbondedForce* f : g.seq) {
					f->ensureForce(topo);
					run.push_back(f->myForce);
				}
			}
		}
		pmgpu_energies_mol e;
		memset(&e, 0, sizeof(e));
		unsigned flags = energies->virial() ? PMGPU_FLAG_VIRIAL : 0u;
		const bool molvir = energies->molecularVirial();
		if (molvir) {
			// the molecule positions the integrator or front end set
			// (buildMolecularCenterOfMass / minimalImage), read as the
			// reference's forces read them
			std::vector<double>& mp = molecule_positions();
			mp.resize(3 * topo->molecules.size());
			for (size_t m = 0; m < topo->molecules.size(); ++m) {
				const Vector3D& c = topo->molecules[m].position;
				mp[3 * m] = c.x; mp[3 * m + 1] = c.y; mp[3 * m + 2] = c.z;
			}
			if (pmgpu_set_molecule_positions(mySystem, (int)topo->molecules.size(), mp.data()) != PMGPU_OK)
				gpu_fail(mySystem, "molecule positions");
			flags |= PMGPU_FLAG_MOLECULAR_VIRIAL;
		}
		int r = pmgpu_evaluate(mySystem, (int)run.size(), run.data(), &((*positions)[0].x), &((*forces)[0].x),
		                       reinterpret_cast<pmgpu_energies*>(&e), flags);
		++g_evaluations;
		if (r != PMGPU_OK) gpu_fail(mySystem, "evaluate");
		// ScalarStructure slots (base/ScalarStructure.h:25-54)
		(*energies)[ScalarStructure::LENNARDJONES] += e.lennard_jones;
		(*energies)[ScalarStructure::COULOMB] += e.coulomb;
		// with the molecular virial alone the atomic slots hold the pairs of
		// different molecules, as ScalarStructure::addVirial(f, d, comDiff) adds them
		if (energies->virial() || molvir) {
			const ScalarStructure::Index v[9] = {ScalarStructure::VIRIALXX, ScalarStructure::VIRIALXY,
			                                     ScalarStructure::VIRIALXZ, ScalarStructure::VIRIALYX,
			                                     ScalarStructure::VIRIALYY, ScalarStructure::VIRIALYZ,
			                                     ScalarStructure::VIRIALZX, ScalarStructure::VIRIALZY,
			                                     ScalarStructure::VIRIALZZ};
			for (int k = 0; k < 9; ++k) (*energies)[v[k]] += e.virial[k];
		}
		if (molvir) {
			const ScalarStructure::Index m[9] = {ScalarStructure::MOLVIRIALXX, ScalarStructure::MOLVIRIALXY,
			                                     ScalarStructure::MOLVIRIALXZ, ScalarStructure::MOLVIRIALYX,
			                                     ScalarStructure::MOLVIRIALYY, ScalarStructure::MOLVIRIALYZ,
			                                     ScalarStructure::MOLVIRIALZX, ScalarStructure::MOLVIRIALZY,
			                                     ScalarStructure::MOLVIRIALZZ};
			for (int k = 0; k < 9; ++k) (*energies)[m[k]] += e.molecular_virial[k];
		}
	}

	// ------------------------------------------------------------ registration
	template <class SW, class P>
	static void reg1(int pot, int sw)
	{
		int p[1] = {pot}, s[1] = {sw};
		ForceFactory::registerExemplar(new GpuNonbondedForce(
			new NonbondedCutoffSystemForce<CubicCellManager, OneAtomPair<PBC, SW, P>>(), 0, 1, p, s,
			GpuNonbondedForce::defaultPrecision()));
	}

	template <class SW1, class SW2, class P2>
	static void reg2(int sw1, int sw2, int pot2)
	{
		int p[2] = {PMGPU_POT_LENNARD_JONES, pot2}, s[2] = {sw1, sw2};
		ForceFactory::registerExemplar(new GpuNonbondedForce(
			new NonbondedCutoffSystemForce<CubicCellManager, OneAtomPairTwo<PBC, SW1, LennardJonesForce, SW2, P2>>(),
			0, 2, p, s, GpuNonbondedForce::defaultPrecision()));
	}

	// a table potential: its tabulated switching function is sw; the pair is Universal
	template <class P>
	static void reg1t(int pot, int sw)
	{
		int p[1] = {pot}, s[1] = {sw};
		ForceFactory::registerExemplar(new GpuNonbondedForce(
			new NonbondedCutoffSystemForce<CubicCellManager, OneAtomPair<PBC, UniversalSwitchingFunction, P>>(), 0, 1,
			p, s, GpuNonbondedForce::defaultPrecision()));
	}

	template <class SW1, class P1, class P2>
	static void reg2t(int pot1, int sw1, int pot2, int sw2)
	{
		int p[2] = {pot1, pot2}, s[2] = {sw1, sw2};
		ForceFactory::registerExemplar(new GpuNonbondedForce(
			new NonbondedCutoffSystemForce<CubicCellManager,
			                               OneAtomPairTwo<PBC, SW1, P1, UniversalSwitchingFunction, P2>>(),
			0, 2, p, s, GpuNonbondedForce::defaultPrecision()));
	}

	template <bool REAL, bool RECIP, bool CORR>
	static void regpme(const std::vector<std::string>& aliases)
	{
		ForceFactory::registerExemplar(new GpuNonbondedForce(
			new NonbondedPMEwaldSystemForce<PBC, CubicCellManager, REAL, RECIP, CORR, BSpline, CutoffSwitchingFunction>(),
			1, 0, NULL, NULL, GpuNonbondedForce::defaultPrecision()), aliases);
	}

	void registerGpuForceExemplars()
	{
		const int LJ = PMGPU_POT_LENNARD_JONES, CO = PMGPU_POT_COULOMB, EW = PMGPU_POT_EWALD_REAL;
		const int C1 = PMGPU_SW_C1, C2 = PMGPU_SW_C2, CUT = PMGPU_SW_CUTOFF, SH = PMGPU_SW_SHIFT;
		// registerForceExemplarsCutoff.cpp:39-67 (single terms)
		reg1<C1SwitchingFunction, CoulombForce>(CO, C1);
		reg1<C2SwitchingFunction, CoulombForce>(CO, C2);
		reg1<CutoffSwitchingFunction, CoulombForce>(CO, CUT);
		reg1<ShiftSwitchingFunction, CoulombForce>(CO, SH);
		reg1<CutoffSwitchingFunction, CoulombEwaldRealForce>(EW, CUT);
		reg1<C1SwitchingFunction, LennardJonesForce>(LJ, C1);
		reg1<C2SwitchingFunction, LennardJonesForce>(LJ, C2);
		reg1<CutoffSwitchingFunction, LennardJonesForce>(LJ, CUT);
		reg1<ShiftSwitchingFunction, LennardJonesForce>(LJ, SH);
		// look-up-table potentials (registerForceExemplarsCutoff.cpp:47-48,58,69)
		typedef LennardJonesTableForce<C2SwitchingFunction, 7, Real> LJT;
		typedef CoulombTableForce<CutoffSwitchingFunction, 6, Real> COTC;
		typedef CoulombTableForce<ShiftSwitchingFunction, 6, Real> COTS;
		typedef CoulombEwaldRealTableForce<CutoffSwitchingFunction, 6, Real> EWT;
		const int LJTP = PMGPU_POT_LENNARD_JONES_TABLE, COTP = PMGPU_POT_COULOMB_TABLE;
		const int EWTP = PMGPU_POT_EWALD_REAL_TABLE;
		reg1t<COTC>(COTP, CUT);
		reg1t<COTS>(COTP, SH);
		reg1t<EWT>(EWTP, CUT);
		reg1t<LJT>(LJTP, C2);
		// LennardJones + CoulombEwaldRealTable (:86,101,132), LennardJonesTable
		// + CoulombEwaldRealTable / CoulombTable (:133-134)
		reg2t<C1SwitchingFunction, LennardJonesForce, EWT>(LJ, C1, EWTP, CUT);
		reg2t<C2SwitchingFunction, LennardJonesForce, EWT>(LJ, C2, EWTP, CUT);
		reg2t<CutoffSwitchingFunction, LennardJonesForce, EWT>(LJ, CUT, EWTP, CUT);
		reg2t<UniversalSwitchingFunction, LJT, EWT>(LJTP, C2, EWTP, CUT);
		reg2t<UniversalSwitchingFunction, LJT, COTS>(LJTP, C2, COTP, SH);
		// registerForceExemplarsCutoff.cpp:76-131 (LennardJones + Coulomb-type pairs)
		reg2<C1SwitchingFunction, CutoffSwitchingFunction, CoulombEwaldRealForce>(C1, CUT, EW);
		reg2<C1SwitchingFunction, ShiftSwitchingFunction, CoulombForce>(C1, SH, CO);
		reg2<C2SwitchingFunction, C1SwitchingFunction, CoulombForce>(C2, C1, CO);
		reg2<C2SwitchingFunction, CutoffSwitchingFunction, CoulombEwaldRealForce>(C2, CUT, EW);
		reg2<C2SwitchingFunction, CutoffSwitchingFunction, CoulombForce>(C2, CUT, CO);
		reg2<C2SwitchingFunction, ShiftSwitchingFunction, CoulombForce>(C2, SH, CO);
		reg2<CutoffSwitchingFunction, CutoffSwitchingFunction, CoulombEwaldRealForce>(CUT, CUT, EW);
		// new: LennardJones Coulomb -switchingFunction C2 -switchingFunction C2 (one fused pass)
		reg2<C2SwitchingFunction, C2SwitchingFunction, CoulombForce>(C2, C2, CO);
		// registerForceExemplarsFastElectrostatic.cpp:50-55; -real runs on the GPU
		// for boxes whose every edge exceeds 2 cutoff (no lattice images)
		std::vector<std::string> none, pme;
		pme.push_back("CoulombPME");
		regpme<true, true, true>(pme);
		regpme<true, false, false>(none);
		regpme<true, false, true>(none);
		regpme<false, true, false>(none);
		regpme<false, true, true>(none);
		regpme<false, false, true>(none);
	}
}
