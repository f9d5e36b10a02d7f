// GpuLinkedCells: see GpuLinkedCells.h. Reference paths are relative to the reference's mardyn/.
#include "GpuLinkedCells.h"

#include <cmath>
#include <cstdlib>

#include "Domain.h"
#include "molecules/Component.h"
#include "molecules/Molecule.h"
#include "particleContainer/adapter/ParticlePairs2PotForceAdapter.h"
#include "utils/Logger.h"

using Log::global_log;

GpuLinkedCells::GpuLinkedCells(ParticlePairsHandler* partPairsHandler, double bBoxMin[3], double bBoxMax[3],
                               double cutoff, double lj_cutoff, Domain* domain, int precision, int device)
    : ParticleContainer(partPairsHandler, bBoxMin, bBoxMax),
      _ctx(nullptr),
      _domain(domain),
      _cutoff(cutoff),
      _ljCutoff(lj_cutoff),
      _n(0),
      _mirrorValid(true),
      _mirrorHandedOut(false),
      _structureChanged(false),
      _iter(0) {
	for (int d = 0; d < 3; d++) {
		if (bBoxMin[d] != 0.0) {
			global_log->error() << "GpuLinkedCells: the bounding box must start at the origin" << std::endl;
			exit(1);
		}
		_L[d] = bBoxMax[d] - bBoxMin[d];
	}
	// single-centre LJ components: one LJ centre at the origin (Component::addLJcenter,
	// molecules/Component.cpp:44-72); the shift flag is a non-zero shift6
	std::vector<Component>& comps = domain->getComponents();
	std::vector<mdgpu_component> mc(comps.size());
	for (size_t i = 0; i < comps.size(); i++) {
		Component& c = comps[i];
		if (c.numLJcenters() != 1 || c.numCharges() || c.numDipoles() || c.numQuadrupoles() || c.numTersoff()) {
			global_log->error() << "GpuLinkedCells: component " << i
			                    << " is not a single LJ centre (use the rigid device container)" << std::endl;
			exit(1);
		}
		const LJcenter& lj = c.ljcenter(0);
		if (lj.rx() != 0.0 || lj.ry() != 0.0 || lj.rz() != 0.0) {
			global_log->error() << "GpuLinkedCells: component " << i << " has its LJ centre off the origin" << std::endl;
			exit(1);
		}
		mc[i].eps = lj.eps();
		mc[i].sigma = lj.sigma();
		mc[i].mass = c.m();
		mc[i].do_shift = lj.shift6() != 0.0 ? 1 : 0;
	}
	// mixing coefficients (xi, eta) of each component pair i < j, InputOldstyle.cpp:206-215
	std::vector<double>& mix = domain->getmixcoeff();
	const int st = mdgpu_create(&_ctx, _L, cutoff, lj_cutoff, 1.0, (int) comps.size(), mc.data(),
	                            mix.empty() ? nullptr : mix.data(), precision, device);
	if (st != MDGPU_OK) fail(st, "mdgpu_create");
	int32_t nc[3];
	double cl[3], hm[3];
	mdgpu_get_geometry(_ctx, nc, cl, hm);
	for (int d = 0; d < 3; d++) _haloL[d] = cl[d];
}

GpuLinkedCells::~GpuLinkedCells() { mdgpu_destroy(_ctx); }

void GpuLinkedCells::fail(int status, const char* where) const {
	global_log->error() << "GpuLinkedCells: " << where << " failed (" << status
	                    << "): " << (_ctx ? mdgpu_last_error(_ctx) : "") << std::endl;
	exit(status);
}

void GpuLinkedCells::rebuild(double bBoxMin[3], double bBoxMax[3]) {
	for (int d = 0; d < 3; d++)
		if (bBoxMin[d] != _boundingBoxMin[d] || bBoxMax[d] != _boundingBoxMax[d]) {
			global_log->error() << "GpuLinkedCells: the box cannot change after construction" << std::endl;
			exit(1);
		}
}

// ---- host mirror -------------------------------------------------------------------------------

void GpuLinkedCells::download() {
	if (_mirrorValid) return;
	std::vector<uint64_t> id(_n);
	std::vector<int32_t> cid(_n);
	std::vector<double> r(3 * _n), v(3 * _n), F(3 * _n);
	const int st = mdgpu_get_particles(_ctx, _n, id.data(), cid.data(), r.data(), v.data(), F.data());
	if (st != MDGPU_OK) fail(st, "mdgpu_get_particles");
	std::vector<Component>* comps = &_domain->getComponents();
	if ((int64_t) _mirror.size() != _n) {
		global_log->error() << "GpuLinkedCells: host mirror out of step with the device" << std::endl;
		exit(1);
	}
	for (int64_t i = 0; i < _n; i++) {
		// orientation and angular momentum of a single-centre molecule do not change (no torque on a
		// centre at the origin): the ones it was loaded with are kept
		const Molecule& old = *_mirror[i];
		Molecule* m = new Molecule(id[i], cid[i], r[3 * i], r[3 * i + 1], r[3 * i + 2], v[3 * i], v[3 * i + 1],
		                           v[3 * i + 2], old.q().qw(), old.q().qx(), old.q().qy(), old.q().qz(), old.D(0),
		                           old.D(1), old.D(2), comps);
		m->setF(&F[3 * i]);
		_mirror[i].reset(m);
	}
	_r0.swap(r);
	_v0.swap(v);
	_F0.swap(F);
	_mirrorValid = true;
	_mirrorHandedOut = false;
}

void GpuLinkedCells::uploadAll() {
	const int64_t n = (int64_t) _mirror.size();
	std::vector<uint64_t> id(n);
	std::vector<int32_t> cid(n);
	std::vector<double> r(3 * n), v(3 * n), F(3 * n);
	for (int64_t i = 0; i < n; i++) {
		const Molecule& m = *_mirror[i];
		id[i] = m.id();
		cid[i] = (int32_t) m.componentid();
		for (int d = 0; d < 3; d++) {
			r[3 * i + d] = m.r(d);
			v[3 * i + d] = m.v(d);
			F[3 * i + d] = m.F(d);
		}
	}
	const int st = mdgpu_set_particles(_ctx, n, id.data(), cid.data(), r.data(), v.data(), F.data());
	if (st != MDGPU_OK) fail(st, "mdgpu_set_particles");
	_n = n;
	_count.assign(_domain->getComponents().size(), 0);
	for (int64_t i = 0; i < n; i++) _count[cid[i]]++;
	_r0.swap(r);
	_v0.swap(v);
	_F0.swap(F);
}

bool GpuLinkedCells::syncToDevice() {
	if (_structureChanged) {
		uploadAll();
		_structureChanged = false;
		_mirrorHandedOut = false;
		return true;
	}
	if (!_mirrorHandedOut) return false;
	_mirrorHandedOut = false;
	bool changed = false;
	for (int64_t i = 0; i < _n && !changed; i++) {
		const Molecule& m = *_mirror[i];
		for (int d = 0; d < 3; d++)
			if (m.r(d) != _r0[3 * i + d] || m.v(d) != _v0[3 * i + d] || m.F(d) != _F0[3 * i + d]) changed = true;
	}
	if (changed) uploadAll();
	return changed;
}

// ---- ParticleContainer -------------------------------------------------------------------------

void GpuLinkedCells::update() {
	syncToDevice();
	const int st = mdgpu_update(_ctx);
	if (st != MDGPU_OK) fail(st, "mdgpu_update");
	_mirrorValid = false;
}

void GpuLinkedCells::addParticle(Molecule& particle) {
	// LinkedCells::addParticle keeps only molecules inside the halo box (LinkedCells.cpp:182-204); the
	// device container holds the box's own molecules, [0, L) after the next update()
	download();
	for (int d = 0; d < 3; d++)
		if (!(particle.r(d) >= -_haloL[d] && particle.r(d) < _L[d] + _haloL[d])) return;
	_mirror.push_back(std::unique_ptr<Molecule>(new Molecule(particle)));
	_structureChanged = true;
}

void GpuLinkedCells::traversePairs() {
	// molecules the host changed since update() are binned again first (uploading invalidates the
	// device's cells)
	if (syncToDevice()) {
		const int su = mdgpu_update(_ctx);
		if (su != MDGPU_OK) fail(su, "mdgpu_update");
	}
	double upot = 0.0, virial = 0.0, npairs = 0.0;
	const int st = mdgpu_traverse_pairs(_ctx, &upot, &virial, &npairs);
	if (st != MDGPU_OK) fail(st, "mdgpu_traverse_pairs");
	// what ParticlePairs2PotForceAdapter::finish stores (single LJ centres: no multipole terms)
	_domain->setLocalVirial(virial);
	_domain->setLocalUpot(upot);
	_mirrorValid = false;
}

unsigned long GpuLinkedCells::getNumberOfParticles() {
	if (_structureChanged) return (unsigned long) _mirror.size();
	return (unsigned long) _n;
}

Molecule* GpuLinkedCells::begin() {
	download();
	_mirrorHandedOut = true;
	_iter = 0;
	return _iter < _mirror.size() ? _mirror[_iter].get() : nullptr;
}

Molecule* GpuLinkedCells::next() {
	_iter++;
	return _iter < _mirror.size() ? _mirror[_iter].get() : nullptr;
}

Molecule* GpuLinkedCells::end() { return nullptr; }

Molecule* GpuLinkedCells::deleteCurrent() {
	if (_iter >= _mirror.size()) return nullptr;
	_mirror.erase(_mirror.begin() + (long) _iter);
	_structureChanged = true;
	return _iter < _mirror.size() ? _mirror[_iter].get() : nullptr;
}

void GpuLinkedCells::deleteOuterParticles() {}

double GpuLinkedCells::get_halo_L(int index) const { return _haloL[index]; }

void GpuLinkedCells::getHaloParticles(std::list<Molecule*>& haloParticlePtrs) { (void) haloParticlePtrs; }

void GpuLinkedCells::getRegion(double lowCorner[3], double highCorner[3], std::list<Molecule*>& particlePtrs) {
	download();
	_mirrorHandedOut = true;
	for (size_t i = 0; i < _mirror.size(); i++) {
		Molecule& m = *_mirror[i];
		bool in = true;
		for (int d = 0; d < 3; d++) in = in && m.r(d) >= lowCorner[d] && m.r(d) < highCorner[d];
		if (in) particlePtrs.push_back(&m);
	}
}

unsigned GpuLinkedCells::countParticles(unsigned int cid) {
	download();
	unsigned n = 0;
	for (size_t i = 0; i < _mirror.size(); i++)
		if (_mirror[i]->componentid() == cid) n++;
	return n;
}

unsigned GpuLinkedCells::countParticles(unsigned int cid, double* cbottom, double* ctop) {
	download();
	unsigned n = 0;
	for (size_t i = 0; i < _mirror.size(); i++) {
		const Molecule& m = *_mirror[i];
		bool in = m.componentid() == cid;
		for (int d = 0; d < 3; d++) in = in && m.r(d) >= cbottom[d] && m.r(d) < ctop[d];
		if (in) n++;
	}
	return n;
}

void GpuLinkedCells::deleteMolecule(unsigned long molid, double x, double y, double z) {
	(void) x;
	(void) y;
	(void) z;
	download();
	for (size_t i = 0; i < _mirror.size(); i++)
		if (_mirror[i]->id() == molid) {
			_mirror.erase(_mirror.begin() + (long) i);
			_structureChanged = true;
			return;
		}
	global_log->error() << "GpuLinkedCells: molecule " << molid << " to delete not found" << std::endl;
	exit(1);
}

double GpuLinkedCells::getEnergy(Molecule* m1) {
	if (m1->numTersoff() > 0) {
		global_log->error() << "The grand canonical ensemble is not implemented for solids." << std::endl;
		exit(484);
	}
	download();
	const double rc2 = _cutoff * _cutoff, rclj2 = _ljCutoff * _ljCutoff;
	double u = 0.0;
	for (size_t i = 0; i < _mirror.size(); i++) {
		Molecule& m2 = *_mirror[i];
		if (m2.id() == m1->id()) continue;
		// the minimum image of m2 seen from m1: dr = r1 - (r2 + shift), as the halo copies give it
		double dr[3], dd = 0.0;
		for (int d = 0; d < 3; d++) {
			double x = m1->r(d) - m2.r(d);
			if (x > 0.5 * _L[d]) x = m1->r(d) - (m2.r(d) + _L[d]);
			else if (x < -0.5 * _L[d]) x = m1->r(d) - (m2.r(d) - _L[d]);
			dr[d] = x;
			dd += x * x;
		}
		if (dd > rc2) continue;
		u += _particlePairsHandler->processPair(*m1, m2, dr, MOLECULE_MOLECULE_FLUID, dd, dd < rclj2);
	}
	return u;
}

int GpuLinkedCells::grandcanonicalBalance(DomainDecompBase* comm) {
	(void) comm;
	return 0;
}

void GpuLinkedCells::grandcanonicalStep(ChemicalPotential* mu, double T) {
	(void) mu;
	(void) T;
	global_log->error() << "GpuLinkedCells: grand-canonical steps are not supported on the device" << std::endl;
	exit(1);
}

// Cell::calcVelocity keeps per-cell velocity sums that nothing on the LJ path reads; the device
// container has no host cells.
void GpuLinkedCells::calcVelocity() {}

// ---- Leapfrog on the device --------------------------------------------------------------------

void GpuLinkedCells::leapfrogPre(double dt, double vcorr) {
	syncToDevice();
	const int st = mdgpu_leapfrog_pre(_ctx, dt, vcorr);
	if (st != MDGPU_OK) fail(st, "mdgpu_leapfrog_pre");
	_mirrorValid = false;
}

double GpuLinkedCells::leapfrogPost(double dtHalf) {
	syncToDevice();
	double summv2 = 0.0;
	const int st = mdgpu_leapfrog_post(_ctx, dtHalf, &summv2);
	if (st != MDGPU_OK) fail(st, "mdgpu_leapfrog_post");
	_mirrorValid = false;
	return summv2;
}
