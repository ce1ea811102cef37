// GpuNonbondedForce.cpp -- see GpuNonbondedForce.h.
#include "Report.h"
using namespace ProtoMol::Report;

#include "GpuNonbondedForce.h"

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
		bool dirty = true;
	};

	static std::map<const GenericTopology*, GpuContext>& contexts()
	{
		static std::map<const GenericTopology*, GpuContext> m;
		return m;
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
		}
		if (c.cell != cell || memcmp(c.box, box, sizeof(box)) != 0) {
			if (pmgpu_set_box(c.sys, box, box + 3, box + 6, box + 9, cell) != PMGPU_OK) gpu_fail(c.sys, "set_box");
			memcpy(c.box, box, sizeof(box));
			c.cell = cell;
		}
		return c;
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
		for (auto& kv : contexts()) kv.second.dirty = true;
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
		if (energies->molecularVirial())
			report << error << "[GpuNonbondedForce] the molecular virial is not computed on the GPU" << endr;
		if (positions->size() == 0) return;
		pmgpu_energies e;
		memset(&e, 0, sizeof(e));
		unsigned flags = energies->virial() ? PMGPU_FLAG_VIRIAL : 0u;
		int r = pmgpu_evaluate(mySystem, 1, &myForce, &((*positions)[0].x), &((*forces)[0].x), &e, flags);
		if (r != PMGPU_OK) gpu_fail(mySystem, "evaluate");
		// ScalarStructure slots (base/ScalarStructure.h:25-54)
		(*energies)[ScalarStructure::LENNARDJONES] += e.lennard_jones;
		(*energies)[ScalarStructure::COULOMB] += e.coulomb;
		if (energies->virial()) {
			const ScalarStructure::Index v[9] = {ScalarStructure::VIRIALXX, ScalarStructure::VIRIALXY,
			                                     ScalarStructure::VIRIALXZ, ScalarStructure::VIRIALYX,
			                                     ScalarStructure::VIRIALYY, ScalarStructure::VIRIALYZ,
			                                     ScalarStructure::VIRIALZX, ScalarStructure::VIRIALZY,
			                                     ScalarStructure::VIRIALZZ};
			for (int k = 0; k < 9; ++k) (*energies)[v[k]] += e.virial[k];
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
