/* -*- c++ -*- */
// GpuNonbondedForce.h -- ProtoMol-side drop-in for the B200 nonbonded path.
//
// A GpuNonbondedForce is a SystemForce (forces/SystemForce.h:18-76) that
// wraps the reference's own force object of the same kind: the wrapped object
// supplies the id (getIdNoAlias), the parameter list (getParameters /
// getParameterSize) and the validation of make() -- so ForceFactory matches,
// parses and rejects exactly what it does for the reference -- and evaluate()
// runs on the GPU through libpmgpu (include/pmgpu.h).
//
// registerGpuForceExemplars() re-registers every periodic NonbondedCutoff
// combination and every PMEwald variant the reference registers
// (factories/registerForceExemplarsCutoff.cpp:36-131,
// factories/registerForceExemplarsFastElectrostatic.cpp:50-55) under the same
// ids; a later registration under an existing id overwrites the earlier one
// (frontend/Factory.h:220-235), so calling it right after
// registerForceExemplars(topo) (applications/protomol-app/protomol.cpp:456)
// makes the unchanged integrators use the GPU forces.
#ifndef GPUNONBONDEDFORCE_H
#define GPUNONBONDEDFORCE_H

#include <string>
#include <vector>

#include "SystemForce.h"
#include "pmgpu.h"

namespace ProtoMol
{
	class GenericTopology;

	class GpuNonbondedForce : public SystemForce
	{
	public:
		// kind 0: NonbondedCutoff (pot/sw describe the OneAtomPair[Two]);
		// kind 1: PMEwald.  'reference' is the wrapped reference force
		// (exemplar or made instance); ownership passes to this object.
		GpuNonbondedForce(SystemForce* reference, int kind, int n_terms, const int* pot, const int* sw,
		                  int precision);
		virtual ~GpuNonbondedForce();

		virtual void evaluate(const GenericTopology* topo, const Vector3DBlock* positions,
		                      Vector3DBlock* forces, ScalarStructure* energies);
		virtual void parallelEvaluate(const GenericTopology* topo, const Vector3DBlock* positions,
		                              Vector3DBlock* forces, ScalarStructure* energies)
		{
			evaluate(topo, positions, forces, energies);
		}
		virtual unsigned int numberOfBlocks(const GenericTopology*, const Vector3DBlock*)
		{
			return 1;
		}
		virtual std::string getKeyword() const;
		virtual void uncache();
		virtual std::string getIdNoAlias() const;
		virtual void getParameters(std::vector<Parameter>& parameters) const;
		virtual unsigned int getParameterSize() const;

		// process-wide default precision of forces made from now on
		// (PMGPU_PRECISION_MIXED unless PMGPU_PRECISION=fp64 is set)
		static int defaultPrecision();

		// the wrapped reference force (its id, parameters and validation)
		const SystemForce* reference() const { return myReference; }

		// pmgpu_evaluate calls made by the GPU forces of this process (one
		// per force group and step once the group is learned)
		static long long evaluations();

	private:
		virtual Force* doMake(std::string& errMsg, std::vector<Value> values) const;
		bool ensureForce(const GenericTopology* topo);

		SystemForce* myReference;
		int myKind, myTerms, myPrecision;
		int myPot[2], mySw[2];
		pmgpu_force* myForce;
		pmgpu_system* mySystem;
	};

	// Registers the GPU exemplars under the reference's ids (periodic
	// boundary conditions, cubic cell manager).
	void registerGpuForceExemplars();
}
#endif /* GPUNONBONDEDFORCE_H */
