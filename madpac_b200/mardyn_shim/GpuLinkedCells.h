// GpuLinkedCells: a MarDyn ParticleContainer (particleContainer/ParticleContainer.h:65-216 of the
// reference's mardyn/ tree) whose molecules live on a B200 and whose update() and traversePairs()
// run there, through the C ABI of libmdgpu.so (include/mdgpu.h). This is the drop-in a MarDyn
// maintainer adds beside LinkedCells; GpuSimulation installs it.
//
// What runs where:
//  * update()        mdgpu_update: periodic wrap and linked-cell binning on the device (the wrap that
//                    exchangeMolecules + deleteOuterParticles perform in the reference, so the
//                    decomposition's exchange is a no-op for this container);
//  * traversePairs() mdgpu_traverse_pairs: forces of all molecules, and Upot and virial, which it
//                    stores with Domain::setLocalUpot / setLocalVirial as
//                    ParticlePairs2PotForceAdapter::finish does (adapter/ParticlePairs2PotForceAdapter.h:64-67);
//  * the Leapfrog transitions run on the device through GpuLeapfrog.
//
// Iteration (begin/next/end, getRegion, countParticles, getEnergy ...) reads a host mirror of the
// molecules, downloaded when first needed after a device operation. The mirror holds each
// molecule's force in F (site forces zero, so calcFM leaves F as it is). Before the next device
// operation the mirror is compared with what was downloaded and whatever the host changed
// (positions, velocities, forces, added or deleted molecules) is uploaded first, so host code that
// modifies molecules through the pointers it is given (thermostat scaling, external forces,
// insertions) stays coherent with the device.
//
// Supported components: single-centre LJ (one LJ centre at the origin, no charges, dipoles,
// quadrupoles or Tersoff centres); others are refused at construction (global_log->error + exit).
// Errors of the device calls follow the reference's convention: global_log->error() and exit(code)
// with the MDGPU_ERR_* code (which mirrors the reference's exit codes where it has one).
#ifndef MADPAC_B200_GPULINKEDCELLS_H_
#define MADPAC_B200_GPULINKEDCELLS_H_

#include <list>
#include <memory>
#include <vector>

#include "mdgpu.h"
#include "particleContainer/ParticleContainer.h"

class Domain;
class Molecule;

class GpuLinkedCells : public ParticleContainer {
public:
	// bBoxMin must be the origin (the device box is [0, bBoxMax)); cutoff and lj_cutoff as
	// LinkedCells takes them; precision MDGPU_FP64 (the drop-in) or MDGPU_MIXED.
	GpuLinkedCells(ParticlePairsHandler* partPairsHandler, double bBoxMin[3], double bBoxMax[3], double cutoff,
	               double lj_cutoff, Domain* domain, int precision = MDGPU_FP64, int device = 0);
	~GpuLinkedCells();

	void rebuild(double bBoxMin[3], double bBoxMax[3]);
	void update();
	void addParticle(Molecule& particle);
	void traversePairs();
	unsigned long getNumberOfParticles();

	Molecule* begin();
	Molecule* next();
	Molecule* end();
	Molecule* deleteCurrent();

	// the device keeps no halo copies: nothing to delete
	void deleteOuterParticles();
	double get_halo_L(int index) const;
	// no halo molecules: the list stays empty
	void getHaloParticles(std::list<Molecule*>& haloParticlePtrs);
	void getRegion(double lowCorner[3], double highCorner[3], std::list<Molecule*>& particlePtrs);
	double getCutoff() { return _cutoff; }
	double getLJCutoff() { return _ljCutoff; }
	double getTersoffCutoff() { return 0.0; }
	unsigned countParticles(unsigned int cid);
	unsigned countParticles(unsigned int cid, double* cbottom, double* ctop);
	void deleteMolecule(unsigned long molid, double x, double y, double z);
	// the molecule's potential energy with every other molecule within the cutoff (minimum image),
	// evaluated by the container's pair handler as LinkedCells::getEnergy does (LinkedCells.cpp:573-617)
	double getEnergy(Molecule* m1);
	// grand-canonical insertion and deletion are not supported on the device container
	int localGrandcanonicalBalance() { return 0; }
	int grandcanonicalBalance(DomainDecompBase* comm);
	void grandcanonicalStep(ChemicalPotential* mu, double T);
	void calcVelocity();

	// ---- device-side operations used by GpuLeapfrog and GpuSimulation --------------------------
	// Leapfrog::transition1to2 for every molecule (Molecule::upd_preF with the same roundings).
	void leapfrogPre(double dt, double vcorr);
	// Leapfrog::transition2to3 for every molecule; returns sum m v^2.
	double leapfrogPost(double dtHalf);
	mdgpu_ctx* context() { return _ctx; }
	// molecules of each component (kept from the last upload; components never change on the device)
	const std::vector<unsigned long>& componentCounts() const { return _count; }
	// Uploads what the host changed in the mirror (called before every device operation); true when
	// something was uploaded.
	bool syncToDevice();

private:
	void fail(int status, const char* where) const;
	void download();
	void uploadAll();

	mdgpu_ctx* _ctx;
	Domain* _domain;
	double _cutoff, _ljCutoff;
	double _L[3];
	double _haloL[3];
	int64_t _n;                       // molecules on the device
	// host copies, in the device's (caller's) order (owned pointers: Molecule has no copy assignment)
	std::vector<std::unique_ptr<Molecule> > _mirror;
	std::vector<double> _r0, _v0, _F0;   // what was downloaded into the mirror
	std::vector<unsigned long> _count;   // molecules per component
	bool _mirrorValid;                // the mirror holds the device state
	bool _mirrorHandedOut;            // pointers into the mirror were given out since the download
	bool _structureChanged;           // molecules were added or deleted on the host
	size_t _iter;
};

#endif  // MADPAC_B200_GPULINKEDCELLS_H_
