// GpuSimulation: MarDyn's Simulation (Simulation.h:80-431 of the reference's mardyn/ tree) with the
// LJ hot path on a B200. The configuration is read by the reference's own code (readConfigFile:
// the components, the mixing rules, the box, the old-style phase space); attachGpu() then moves the
// molecules the reference container read into a GpuLinkedCells and installs GpuLeapfrog and
// GpuDomainDecomp in place of the reference's LinkedCells, Leapfrog and DomainDecompDummy, through
// the protected members Simulation gives its subclasses (the way MarDynSimulation, coupling/
// MarDynSimulation.h:30, extends Simulation). Everything else -- prepare_start, simulate and its
// steps, the Domain's global values and thermostat, checkpoints, output plugins -- is the
// reference's unmodified code calling the device through the container and integrator interfaces.
#ifndef MADPAC_B200_GPUSIMULATION_H_
#define MADPAC_B200_GPUSIMULATION_H_

#include "GpuLinkedCells.h"
#include "Simulation.h"
#include "parallel/DomainDecompDummy.h"

// The single-process decomposition with the molecule exchange left to the device container:
// GpuLinkedCells::update() wraps positions into the box and the pair kernels find periodic images
// themselves, so no halo copies are made (DomainDecompDummy::exchangeMolecules,
// parallel/DomainDecompDummy.cpp:22-116, would add them through addParticle).
class GpuDomainDecomp : public DomainDecompDummy {
public:
	void exchangeMolecules(ParticleContainer* moleculeContainer, const std::vector<Component>& components,
	                       Domain* domain);
	void balanceAndExchange(bool balance, ParticleContainer* moleculeContainer, const std::vector<Component>& components,
	                        Domain* domain);
};

class GpuSimulation : public Simulation {
public:
	GpuSimulation();
	// After readConfigFile: the molecules go to the device (MDGPU_FP64, the drop-in, or MDGPU_MIXED)
	// and the device container, integrator and decomposition replace the reference's.
	void attachGpu(int precision = MDGPU_FP64, int device = 0);
	GpuLinkedCells* gpuContainer() { return dynamic_cast<GpuLinkedCells*>(_moleculeContainer); }
	ParticleContainer* container() { return _moleculeContainer; }
};

#endif  // MADPAC_B200_GPUSIMULATION_H_
