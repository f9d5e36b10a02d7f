// GpuLeapfrog: MarDyn's Leapfrog integrator (integrators/Leapfrog.cpp:14-108 of the reference's
// mardyn/ tree, interface integrators/Integrator.h:31-93) with the same three-state machine, whose
// transitions run on the device when the container is a GpuLinkedCells:
//  * eventNewTimestep (state 3 -> 1 -> 2): Molecule::upd_preF(dt, vcorr, Dcorr) for every molecule,
//    vcorr = 2 - 1/beta_trans (Leapfrog::transition1to2), through mdgpu_leapfrog_pre;
//  * eventForcesCalculated (state 2 -> 3): Molecule::upd_postF(dt/2) for every molecule through
//    mdgpu_leapfrog_post, and the sums Leapfrog::transition2to3 hands to the Domain (sum m v^2,
//    sum I w^2 = 0 and no rotational degrees of freedom for single LJ centres, N).
// With another container, or with several thermostats (per-thermostat sums), it iterates the
// molecules on the host exactly as Leapfrog does.
#ifndef MADPAC_B200_GPULEAPFROG_H_
#define MADPAC_B200_GPULEAPFROG_H_

#include "integrators/Integrator.h"

class Leapfrog;

class GpuLeapfrog : public Integrator {
public:
	explicit GpuLeapfrog(double timestepLength);
	~GpuLeapfrog();

	void eventForcesCalculated(ParticleContainer* moleculeContainer, Domain* domain);
	void eventNewTimestep(ParticleContainer* moleculeContainer, Domain* domain);
	// uniform acceleration and z-oscillators act on host molecules (as Leapfrog, which leaves the
	// first two empty and has no oscillators): not used on the LJ path
	void accelerateUniformly(ParticleContainer* molCont, Domain* domain);
	void accelerateInstantaneously(ParticleContainer* molCont, Domain* domain);
	void init1D(unsigned zoscillator, ParticleContainer* molCont);
	void zOscillation(unsigned zoscillator, ParticleContainer* molCont);

private:
	void transition1to2(ParticleContainer* molCont, Domain* domain);
	void transition2to3(ParticleContainer* molCont, Domain* domain);
	Leapfrog* _host;   // the reference's integrator for the host paths
	int _state;
};

#endif  // MADPAC_B200_GPULEAPFROG_H_
