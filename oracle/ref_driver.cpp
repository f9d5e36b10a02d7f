// Test harness around the reference MarDyn sources (compiled unmodified by oracle/Makefile).
//
// It runs exactly the reference's own step sequence -- Simulation::prepare_start
// (mardyn/Simulation.cpp:907-993) followed by Simulation::simulateStep
// (mardyn/Simulation.cpp:1218-1229) -- on an old-style .cfg/.inp pair and records, per step:
//   * the local potential energy and virial that ParticlePairs2PotForceAdapter::finish
//     stored in Domain (mardyn/particleContainer/adapter/ParticlePairs2PotForceAdapter.h:64-67),
//   * sum m v^2 over the molecules,
// and, for the steps named on the command line, every molecule's id, component, r, v, F and
// LinkedCells cell index (LinkedCells::getCellIndexOfMolecule, LinkedCells.cpp:535-547), and in a
// second file its orientation q, angular momentum D and torque M (Molecule::q/D/M,
// molecules/Molecule.h:85-89); rot.txt holds sum I w^2 per step (Molecule::calculate_mv2_Iw2).
//
// The reference never prints per-molecule forces, so this harness exists only to pin the
// oracle and the GPU path against the reference itself. It is test infrastructure.
//
// usage: ref_driver <cfg> <nsteps> <outdir> <dumpsteps: comma list, 0 = after prepare_start>
//        ref_driver --time <cfg> <nsteps>      (timing only: prints seconds per step as JSON)
//        ref_driver --checkpoint <cfg> <nsteps> <file> <outdir>   (the reference's checkpoint after
//                   nsteps steps, and the exact state of that step)
//        ref_driver --time-checkpoint <cfg> <file>   (seconds to write the initial state's checkpoint)
//        ref_driver --farfield <cfg>   (Domain::initFarFieldCorr's _UpotCorr and _VirialCorr as JSON)
#include <sys/time.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <sstream>
#include <string>
#include <vector>

// getCellIndexOfMolecule is private in LinkedCells and the far-field terms are private in Domain;
// the harness reads them directly.
#define private public
#include "particleContainer/LinkedCells.h"
#include "Domain.h"
#undef private

#include "Simulation.h"
#include "coupling/boundary/ForceBoundary.h"
#include "coupling/boundary/ReflectingBoundary.h"
#include "molecules/Molecule.h"
#include "parallel/DomainDecompBase.h"
#include "particleContainer/ParticleContainer.h"
#include "utils/Logger.h"

using Log::global_log;

namespace {

double now_s() {
	struct timeval tv;
	gettimeofday(&tv, nullptr);
	return tv.tv_sec + 1e-6 * tv.tv_usec;
}

struct Rec {
	unsigned long id;
	long cid;
	double r[3], v[3], F[3];
	long cell;
	double q[4], D[3], M[3];
};

}  // namespace

class RefDriver : public Simulation {
public:
	Domain* domain() { return _domain; }

	double summv2() {
		double s = 0.0;
		for (Molecule* m = _moleculeContainer->begin(); m != _moleculeContainer->end(); m = _moleculeContainer->next()) {
			double v2 = m->v(0) * m->v(0) + m->v(1) * m->v(1) + m->v(2) * m->v(2);
			s += m->getMass() * v2;
		}
		return s;
	}

	void writeScalars(FILE* f, long step) {
		fprintf(f, "%ld %.17g %.17g %.17g %lu\n", step, _domain->getLocalUpot(), _domain->getLocalVirial(), summv2(),
		        _moleculeContainer->getNumberOfParticles());
	}

	void writeRot(FILE* f, long step) {
		double mv2 = 0.0, iw2 = 0.0;
		for (Molecule* m = _moleculeContainer->begin(); m != _moleculeContainer->end(); m = _moleculeContainer->next())
			m->calculate_mv2_Iw2(mv2, iw2);
		fprintf(f, "%ld %.17g\n", step, iw2);
	}

	void writeArrays(const std::string& outdir, long step) {
		LinkedCells* lc = dynamic_cast<LinkedCells*>(_moleculeContainer);
		std::vector<Rec> recs;
		for (Molecule* m = _moleculeContainer->begin(); m != _moleculeContainer->end(); m = _moleculeContainer->next()) {
			Rec r;
			r.id = m->id();
			r.cid = m->componentid();
			for (int d = 0; d < 3; d++) {
				r.r[d] = m->r(d);
				r.v[d] = m->v(d);
				r.F[d] = m->F(d);
			}
			r.cell = lc ? (long) lc->getCellIndexOfMolecule(m) : -1;
			r.q[0] = m->q().qw();
			r.q[1] = m->q().qx();
			r.q[2] = m->q().qy();
			r.q[3] = m->q().qz();
			for (int d = 0; d < 3; d++) {
				r.D[d] = m->D(d);
				r.M[d] = m->M(d);
			}
			recs.push_back(r);
		}
		std::sort(recs.begin(), recs.end(), [](const Rec& a, const Rec& b) { return a.id < b.id; });
		char name[512];
		snprintf(name, sizeof(name), "%s/step%06ld.bin", outdir.c_str(), step);
		FILE* f = fopen(name, "wb");
		if (!f) {
			fprintf(stderr, "cannot open %s\n", name);
			std::exit(2);
		}
		long n = (long) recs.size();
		fwrite(&n, sizeof(long), 1, f);
		for (const Rec& r : recs) fwrite(&r.id, sizeof(unsigned long), 1, f);
		for (const Rec& r : recs) fwrite(&r.cid, sizeof(long), 1, f);
		for (const Rec& r : recs) fwrite(r.r, sizeof(double), 3, f);
		for (const Rec& r : recs) fwrite(r.v, sizeof(double), 3, f);
		for (const Rec& r : recs) fwrite(r.F, sizeof(double), 3, f);
		for (const Rec& r : recs) fwrite(&r.cell, sizeof(long), 1, f);
		fclose(f);
		snprintf(name, sizeof(name), "%s/step%06ld.rot.bin", outdir.c_str(), step);
		f = fopen(name, "wb");
		if (!f) {
			fprintf(stderr, "cannot open %s\n", name);
			std::exit(2);
		}
		fwrite(&n, sizeof(long), 1, f);
		for (const Rec& r : recs) fwrite(r.q, sizeof(double), 4, f);
		for (const Rec& r : recs) fwrite(r.D, sizeof(double), 3, f);
		for (const Rec& r : recs) fwrite(r.M, sizeof(double), 3, f);
		fclose(f);
	}

	void run(unsigned long nsteps, const std::string& outdir, const std::set<long>& dumps) {
		std::string sname = outdir + "/scalars.txt";
		FILE* sf = fopen(sname.c_str(), "w");
		std::string rname = outdir + "/rot.txt";
		FILE* rf = fopen(rname.c_str(), "w");
		prepare_start();
		writeScalars(sf, 0);
		writeRot(rf, 0);
		if (dumps.count(0)) writeArrays(outdir, 0);
		// Simulation::simulate runs _simstep = _initSimulation .. _numberOfTimesteps inclusive;
		// simulateStart sets _initSimulation (Simulation.cpp:1011), so it comes first.
		simulateStart();
		_numberOfTimesteps = _initSimulation + nsteps - 1;
		long k = 1;
		for (_simstep = _initSimulation; _simstep <= _numberOfTimesteps; k++) {
			simulateStep();
			writeScalars(sf, k);
			writeRot(rf, k);
			if (dumps.count(k)) writeArrays(outdir, k);
		}
		fclose(sf);
		fclose(rf);
	}

	// nsteps steps, then the reference's own checkpoint (Domain::writeCheckpoint, Domain.cpp:462-568)
	// and the exact state of that step (writeArrays)
	void checkpoint(unsigned long nsteps, const std::string& path, const std::string& outdir) {
		prepare_start();
		simulateStart();
		_numberOfTimesteps = _initSimulation + nsteps - 1;
		for (_simstep = _initSimulation; _simstep <= _numberOfTimesteps;) simulateStep();
		_domain->writeCheckpoint(path, _moleculeContainer, _domainDecomposition);
		writeArrays(outdir, (long) nsteps);
	}

	// seconds to write the checkpoint of the initial state (after prepare_start)
	double timeCheckpoint(const std::string& path) {
		prepare_start();
		double t0 = now_s();
		_domain->writeCheckpoint(path, _moleculeContainer, _domainDecomposition);
		return now_s() - t0;
	}

	// The molecule-side boundaries of MaDPaC's coupled step (coupling/MarDynSimulation.cpp:61-160)
	// on the configuration as read (molecules placed outside the box stand for those that left it
	// in the drift): the container is binned, ReflectingBoundary::applyBoundary runs (step 1 dump:
	// r, v after it), the pair forces follow with the decomposition's halo copies (step 2 dump), then
	// ForceBoundary::applyBoundary (step 3 dump); calcfm.txt samples ForceBoundary::calcFm.
	void boundary(int dim, int stream_out_dir, int stream_out, const std::string& outdir, const std::string& moves) {
		using madpac::mardyncoupling::boundary::ForceBoundary;
		using madpac::mardyncoupling::boundary::ReflectingBoundary;
		// new positions "id x y z" (outside the box) for some molecules: the reader itself drops
		// molecules outside the box, so they are moved after reading
		FILE* mf = fopen(moves.c_str(), "r");
		unsigned long mid;
		double mx, my, mz;
		while (mf && fscanf(mf, "%lu %lf %lf %lf", &mid, &mx, &my, &mz) == 4)
			for (Molecule* m = _moleculeContainer->begin(); m != _moleculeContainer->end(); m = _moleculeContainer->next())
				if (m->id() == mid) {
					m->setr(0, mx);
					m->setr(1, my);
					m->setr(2, mz);
				}
		if (mf) fclose(mf);
		_moleculeContainer->update();
		ReflectingBoundary rb(_moleculeContainer, _domain, stream_out_dir, false, dim, stream_out != 0);
		rb.applyBoundary();
		writeArrays(outdir, 1);
		_domainDecomposition->balanceAndExchange(true, _moleculeContainer, _domain->getComponents(), _domain);
		_moleculeContainer->traversePairs();
		_moleculeContainer->deleteOuterParticles();
		writeArrays(outdir, 2);
		ForceBoundary fb(_moleculeContainer, _domain, _moleculeContainer->getCutoff(), stream_out_dir, dim);
		fb.applyBoundary();
		writeArrays(outdir, 3);
		FILE* f = fopen((outdir + "/calcfm.txt").c_str(), "w");
		for (int k = 0; k <= 400; k++) {
			const double r = 0.0075 * k;
			fprintf(f, "%.17g %.17g\n", r, ForceBoundary::calcFm(r));
		}
		fclose(f);
	}

	double timeSteps(unsigned long nsteps) {
		prepare_start();
		simulateStart();
		_numberOfTimesteps = _initSimulation + nsteps - 1;
		double t0 = now_s();
		for (_simstep = _initSimulation; _simstep <= _numberOfTimesteps;) simulateStep();
		return (now_s() - t0) / nsteps;
	}
};

int main(int argc, char** argv) {
	global_log = new Log::Logger(Log::MARDYN_Error);
	if (argc >= 4 && std::string(argv[1]) == "--time") {
		RefDriver sim;
		sim.readConfigFile(argv[2]);
		unsigned long n = strtoul(argv[3], nullptr, 10);
		double s = sim.timeSteps(n);
		printf("{\"seconds_per_step\": %.9g, \"steps\": %lu}\n", s, n);
		return 0;
	}
	if (argc >= 6 && std::string(argv[1]) == "--checkpoint") {
		RefDriver sim;
		sim.readConfigFile(argv[2]);
		sim.checkpoint(strtoul(argv[3], nullptr, 10), argv[4], argv[5]);
		return 0;
	}
	if (argc >= 3 && std::string(argv[1]) == "--farfield") {
		RefDriver sim;
		sim.readConfigFile(argv[2]);
		printf("{\"upot_corr\": %.17g, \"virial_corr\": %.17g}\n", sim.domain()->_UpotCorr,
		       sim.domain()->_VirialCorr);
		return 0;
	}
	if (argc >= 8 && std::string(argv[1]) == "--boundary") {
		RefDriver sim;
		sim.readConfigFile(argv[2]);
		sim.boundary(atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), argv[6], argv[7]);
		return 0;
	}
	if (argc >= 4 && std::string(argv[1]) == "--time-checkpoint") {
		RefDriver sim;
		sim.readConfigFile(argv[2]);
		double s = sim.timeCheckpoint(argv[3]);
		printf("{\"seconds\": %.9g}\n", s);
		return 0;
	}
	if (argc < 5) {
		fprintf(stderr, "usage: ref_driver <cfg> <nsteps> <outdir> <dumpsteps>\n");
		return 1;
	}
	std::set<long> dumps;
	std::stringstream ss(argv[4]);
	std::string tok;
	while (std::getline(ss, tok, ','))
		if (!tok.empty()) dumps.insert(strtol(tok.c_str(), nullptr, 10));
	RefDriver sim;
	sim.readConfigFile(argv[1]);
	sim.run(strtoul(argv[2], nullptr, 10), argv[3], dumps);
	return 0;
}
