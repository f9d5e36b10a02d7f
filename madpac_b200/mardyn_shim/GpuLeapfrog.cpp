// GpuLeapfrog: see GpuLeapfrog.h. Reference paths are relative to the reference's mardyn/.
#include "GpuLeapfrog.h"

#include <vector>

#include "Domain.h"
#include "GpuLinkedCells.h"
#include "integrators/Leapfrog.h"
#include "utils/Logger.h"

using Log::global_log;

namespace {

// The device path applies when the container is on the device and one thermostat covers every
// component (Leapfrog::transition2to3 keeps per-thermostat sums otherwise).
GpuLinkedCells* device_container(ParticleContainer* molCont, Domain* domain) {
	GpuLinkedCells* g = dynamic_cast<GpuLinkedCells*>(molCont);
	return (g && !domain->severalThermostats()) ? g : nullptr;
}

}  // namespace

// The host paths (other containers, several thermostats, uniform acceleration, z-oscillators) are
// the reference's own Leapfrog, held by GpuLeapfrog and given every event the device path does not
// take.
GpuLeapfrog::GpuLeapfrog(double timestepLength) : _host(new Leapfrog(timestepLength)), _state(3) {
	_timestepLength = timestepLength;
}

GpuLeapfrog::~GpuLeapfrog() { delete _host; }

void GpuLeapfrog::eventNewTimestep(ParticleContainer* molCont, Domain* domain) {
	if (!device_container(molCont, domain)) {
		_host->eventNewTimestep(molCont, domain);
		return;
	}
	// Leapfrog::eventNewTimestep: state 3 -> 1 (transition3to1) -> 2 (transition1to2)
	if (_state == 3) {
		_state = 1;
		transition1to2(molCont, domain);
	}
}

void GpuLeapfrog::eventForcesCalculated(ParticleContainer* molCont, Domain* domain) {
	if (!device_container(molCont, domain)) {
		_host->eventForcesCalculated(molCont, domain);
		return;
	}
	if (_state == 2) transition2to3(molCont, domain);
}

void GpuLeapfrog::transition1to2(ParticleContainer* molCont, Domain* domain) {
	if (_state != 1) {
		global_log->error() << "GpuLeapfrog::transition1to2(...): Wrong state for state transition" << std::endl;
		return;
	}
	// the velocity correction of the thermostat, as Leapfrog::transition1to2 (Leapfrog.cpp:37-51);
	// single centres have no rotation, so the angular-momentum correction is not needed
	const double vcorr = 2. - 1. / domain->getGlobalBetaTrans();
	device_container(molCont, domain)->leapfrogPre(_timestepLength, vcorr);
	_state = 2;
}

void GpuLeapfrog::transition2to3(ParticleContainer* molCont, Domain* domain) {
	if (_state != 2) {
		global_log->error() << "GpuLeapfrog::transition2to3(...): Wrong state for state transition" << std::endl;
		return;
	}
	GpuLinkedCells* g = device_container(molCont, domain);
	const double summv2 = g->leapfrogPost(0.5 * _timestepLength);
	// the sums Leapfrog::transition2to3 hands to the Domain (Leapfrog.cpp:53-99), thermostat 0
	unsigned long rotDOF = 0;
	const std::vector<unsigned long>& count = g->componentCounts();
	for (size_t c = 0; c < count.size(); c++) rotDOF += count[c] * domain->getComponentRotDOF((int) c);
	domain->setLocalSummv2(summv2, 0);
	domain->setLocalSumIw2(0.0, 0);
	domain->setLocalNrotDOF(0, g->getNumberOfParticles(), rotDOF);
	_state = 3;
}

void GpuLeapfrog::accelerateUniformly(ParticleContainer* molCont, Domain* domain) {
	_host->accelerateUniformly(molCont, domain);
}

void GpuLeapfrog::accelerateInstantaneously(ParticleContainer* molCont, Domain* domain) {
	_host->accelerateInstantaneously(molCont, domain);
}

void GpuLeapfrog::init1D(unsigned zoscillator, ParticleContainer* molCont) {
	_host->init1D(zoscillator, molCont);
}

void GpuLeapfrog::zOscillation(unsigned zoscillator, ParticleContainer* molCont) {
	_host->zOscillation(zoscillator, molCont);
}
