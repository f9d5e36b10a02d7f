// GpuSimulation: see GpuSimulation.h. Reference paths are relative to the reference's mardyn/.
#include "GpuSimulation.h"

#include <cstdlib>

#include "Domain.h"
#include "GpuLeapfrog.h"
#include "molecules/Molecule.h"
#include "utils/Logger.h"

using Log::global_log;

void GpuDomainDecomp::exchangeMolecules(ParticleContainer* moleculeContainer, const std::vector<Component>& components,
                                        Domain* domain) {
	(void) moleculeContainer;
	(void) components;
	(void) domain;
}

void GpuDomainDecomp::balanceAndExchange(bool balance, ParticleContainer* moleculeContainer,
                                         const std::vector<Component>& components, Domain* domain) {
	(void) balance;
	exchangeMolecules(moleculeContainer, components, domain);
}

GpuSimulation::GpuSimulation() : Simulation() {}

void GpuSimulation::attachGpu(int precision, int device) {
	if (dynamic_cast<GpuLinkedCells*>(_moleculeContainer)) return;
	if (!_moleculeContainer || !_integrator || !_domainDecomposition) {
		global_log->error() << "GpuSimulation::attachGpu: read the configuration first" << std::endl;
		exit(1);
	}
	double bMin[3], bMax[3];
	for (int d = 0; d < 3; d++) {
		bMin[d] = _moleculeContainer->getBoundingBoxMin(d);
		bMax[d] = _moleculeContainer->getBoundingBoxMax(d);
	}
	GpuLinkedCells* gpu = new GpuLinkedCells(_particlePairsHandler, bMin, bMax, _moleculeContainer->getCutoff(),
	                                         _moleculeContainer->getLJCutoff(), _domain, precision, device);
	// the molecules the reference's reader placed in its container (no halo copies exist before the
	// first exchange), in its iteration order
	for (Molecule* m = _moleculeContainer->begin(); m != _moleculeContainer->end(); m = _moleculeContainer->next())
		gpu->addParticle(*m);
	delete _moleculeContainer;
	_moleculeContainer = gpu;
	const double dt = _integrator->getTimestepLength();
	delete _integrator;
	_integrator = new GpuLeapfrog(dt);
	delete _domainDecomposition;
	_domainDecomposition = new GpuDomainDecomp();
}
