// Test harness of the MarDyn shim (not part of the shim): runs the reference's own
// Simulation::prepare_start and simulate step sequence (Simulation.cpp:907-1229 of the reference's
// mardyn/ tree) with GpuSimulation's device container, integrator and decomposition on an old-style
// .cfg/.inp pair, and records per step what oracle/ref_driver.cpp records for the reference itself:
// local Upot and virial from the Domain, sum m v^2 over the molecules (iterated through the
// container), and for the steps named on the command line each molecule's id, component, r, v and F
// in the same binary layout (cell index -1: the device container has no host cells). The loop is
// the one Simulation::simulate runs (simulateStart, simulateStep until _numberOfTimesteps,
// simulateFinish, which also writes the reference's final checkpoint).
//
// usage: shim_driver <cfg> <nsteps> <outdir> <dumpsteps: comma list, 0 = after prepare_start> [fp64|mixed]
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "Domain.h"
#include "GpuSimulation.h"
#include "molecules/Molecule.h"
#include "utils/Logger.h"

using Log::global_log;

class ShimDriver : public GpuSimulation {
public:
	double summv2() {
		double s = 0.0;
		for (Molecule* m = _moleculeContainer->begin(); m != _moleculeContainer->end(); m = _moleculeContainer->next())
			s += m->getMass() * (m->v(0) * m->v(0) + m->v(1) * m->v(1) + m->v(2) * m->v(2));
		return s;
	}

	void writeScalars(FILE* f, long step) {
		fprintf(f, "%ld %.17g %.17g %.17g %lu\n", step, _domain->getLocalUpot(), _domain->getLocalVirial(), summv2(),
		        _moleculeContainer->getNumberOfParticles());
	}

	void writeArrays(const std::string& outdir, long step) {
		struct Rec {
			unsigned long id;
			long cid;
			double r[3], v[3], F[3];
		};
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
			recs.push_back(r);
		}
		std::sort(recs.begin(), recs.end(), [](const Rec& a, const Rec& b) { return a.id < b.id; });
		char name[512];
		snprintf(name, sizeof(name), "%s/step%06ld.bin", outdir.c_str(), step);
		FILE* f = fopen(name, "wb");
		if (!f) {
			fprintf(stderr, "cannot open %s\n", name);
			exit(2);
		}
		const long n = (long) recs.size(), none = -1;
		fwrite(&n, sizeof(long), 1, f);
		for (const Rec& r : recs) fwrite(&r.id, sizeof(unsigned long), 1, f);
		for (const Rec& r : recs) fwrite(&r.cid, sizeof(long), 1, f);
		for (const Rec& r : recs) fwrite(r.r, sizeof(double), 3, f);
		for (const Rec& r : recs) fwrite(r.v, sizeof(double), 3, f);
		for (const Rec& r : recs) fwrite(r.F, sizeof(double), 3, f);
		for (long i = 0; i < n; i++) fwrite(&none, sizeof(long), 1, f);
		fclose(f);
	}

	void run(unsigned long nsteps, const std::string& outdir, const std::set<long>& dumps) {
		FILE* sf = fopen((outdir + "/scalars.txt").c_str(), "w");
		prepare_start();
		writeScalars(sf, 0);
		if (dumps.count(0)) writeArrays(outdir, 0);
		simulateStart();
		_numberOfTimesteps = _initSimulation + nsteps - 1;
		long k = 1;
		for (_simstep = _initSimulation; _simstep <= _numberOfTimesteps; k++) {
			simulateStep();
			writeScalars(sf, k);
			if (dumps.count(k)) writeArrays(outdir, k);
		}
		fclose(sf);
		simulateFinish();
	}
};

int main(int argc, char** argv) {
	global_log = new Log::Logger(Log::MARDYN_Error);
	if (argc < 5) {
		fprintf(stderr, "usage: shim_driver <cfg> <nsteps> <outdir> <dumpsteps> [fp64|mixed]\n");
		return 1;
	}
	const int precision = argc > 5 && std::string(argv[5]) == "mixed" ? MDGPU_MIXED : MDGPU_FP64;
	std::set<long> dumps;
	std::stringstream ss(argv[4]);
	std::string tok;
	while (std::getline(ss, tok, ','))
		if (!tok.empty()) dumps.insert(strtol(tok.c_str(), nullptr, 10));
	ShimDriver sim;
	sim.readConfigFile(argv[1]);
	sim.attachGpu(precision, 0);
	sim.run(strtoul(argv[2], nullptr, 10), argv[3], dumps);
	return 0;
}
