// MarDyn old-style phase-space files on the device path: the checkpoint writer and the reader, so
// that a run on the GPU context starts from and ends in the reference's own files without a host
// Molecule container.
//
//   mdgpu_write_checkpoint   Domain::writeCheckpoint (Domain.cpp:462-568) followed by
//                            DomainDecompDummy::writeMoleculesToFile / Molecule::write
//                            (parallel/DomainDecompDummy.cpp:144-154, molecules/Molecule.cpp:263-270)
//   mdgpu_read_phase_space   InputOldstyle::readPhaseSpaceHeader + readPhaseSpace
//                            (io/InputOldstyle.cpp:35-392) for single-site LJ components
//
// Layout of a checkpoint, as the reference's streams print it: the header lines with the
// stream's default precision (6 significant digits) for currentTime and 9 from Length on
// (setprecision(9) is sticky), the component blocks (Component::write, molecules/Component.cpp:170-195;
// LJcenter::write prints x y z, m, eps sigma rc and the centre's shift6 value, molecules/Site.h:109-111),
// the mixing coefficients with the reference's separators and epsilonRF, then one line per
// molecule at 6 significant digits: id, component (1-based), r, v, the unit quaternion, D = 0.
// A C++ stream of precision p prints a double as printf's "%.<p>g", which this file uses. The
// reference writes the molecules in its container's order; this writer uses the caller's order.
// digits > 6 writes the molecule lines at more digits (17: the exact doubles, for restarts).
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "md_internal.h"

namespace mdgpu {
namespace {

constexpr const char* kCheckpointVersion = "20100321";   // Domain.h:31, VERSION

int io_fail(Context* c, int code, const std::string& msg) {
	c->err = msg;
	return code;
}

std::string gfmt(double x, int digits) {
	char b[64];
	snprintf(b, sizeof(b), "%.*g", digits, x);
	return b;
}

unsigned worker_count(int64_t items) {
	unsigned hw = std::thread::hardware_concurrency();
	if (hw == 0) hw = 4;
	const int64_t per = 65536;   // below this a thread is not worth starting
	return (unsigned) std::max<int64_t>(1, std::min<int64_t>(hw, (items + per - 1) / per));
}

// Runs f(k, lo, hi) on [0, n) split into `parts` contiguous ranges, one thread each.
template <typename F>
void parallel_ranges(int64_t n, unsigned parts, F&& f) {
	std::vector<std::thread> th;
	for (unsigned k = 0; k < parts; k++) {
		const int64_t lo = n * k / parts, hi = n * (k + 1) / parts;
		if (k + 1 == parts)
			f(k, lo, hi);
		else
			th.emplace_back([&f, k, lo, hi] { f(k, lo, hi); });
	}
	for (auto& t : th) t.join();
}

std::string checkpoint_header(const Context* c, int64_t n, double current_time, double temperature,
                              double epsilon_rf) {
	std::string h = std::string("mardyn trunk ") + kCheckpointVersion + "\n";
	h += " currentTime\t" + gfmt(current_time, 6) + "\n";
	h += " Length\t" + gfmt(c->g.L[0], 9) + " " + gfmt(c->g.L[1], 9) + " " + gfmt(c->g.L[2], 9) + "\n";
	h += " Temperature\t" + gfmt(temperature, 9) + "\n";
	const int nc = c->sp.n;
	h += " NumberOfComponents\t" + std::to_string(nc) + "\n";
	for (int i = 0; i < nc; i++) {
		h += "1\t0\t0\t0\t0\n";
		h += gfmt(0.0, 9) + " " + gfmt(0.0, 9) + " " + gfmt(0.0, 9) + "\t" + gfmt(c->sp.mass[i], 9) + "\t" +
		     gfmt(c->eps[i], 9) + " " + gfmt(c->sigma[i], 9) + " " + gfmt(c->rc_lj, 9) + " " +
		     gfmt(c->sp.shift6[i * nc + i], 9) + "\n";
		h += gfmt(0.0, 9) + " " + gfmt(0.0, 9) + " " + gfmt(0.0, 9) + "\n";
	}
	// Domain::writeCheckpoint's mixing-coefficient loop: xi eta pairs, a tab between pairs, a line
	// break after each row of the upper triangle, then epsilonRF
	unsigned numperline = (unsigned) nc, iout = 0;
	for (int k = 0; k < nc * (nc - 1); k++) {
		h += gfmt(c->mix[k], 9);
		iout++;
		if (iout / 2 >= numperline) {
			h += "\n";
			iout = 0;
			--numperline;
		} else if (!(iout % 2)) {
			h += "\t";
		} else {
			h += " ";
		}
	}
	h += gfmt(epsilon_rf, 9) + "\n";
	h += " NumberOfMolecules\t" + std::to_string(n) + "\n";
	h += " MoleculeFormat\tICRVQD\n";
	return h;
}

// ---- reader ----------------------------------------------------------------------------------

struct Cursor {
	const char* p;
	const char* end;
	bool token(std::string& t) {
		while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
		if (p >= end) return false;
		const char* s = p;
		while (p < end && !(*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
		t.assign(s, p);
		return true;
	}
	bool number(double& x) {
		std::string t;
		if (!token(t)) return false;
		char* e = nullptr;
		x = strtod(t.c_str(), &e);
		return e && *e == '\0';
	}
};

bool close_to(double a, double b) { return std::fabs(a - b) <= 1e-8 * std::max(std::fabs(a), std::fabs(b)) + 1e-300; }

}  // namespace
}  // namespace mdgpu

using mdgpu::Context;

int mdgpu_write_checkpoint(mdgpu_ctx* ctx, const char* path, double current_time, double temperature,
                           double epsilon_rf, int digits) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (!path) return mdgpu::io_fail(c, MDGPU_ERR_ARG, "path is required");
	if (c->n == 0) return mdgpu::io_fail(c, MDGPU_ERR_STATE, "no molecules loaded");
	if (digits == 0) digits = 6;
	if (digits < 1 || digits > 17) return mdgpu::io_fail(c, MDGPU_ERR_ARG, "digits must be 0 (reference: 6) or 1..17");
	const int64_t n = c->n;
	std::vector<uint64_t> id(n);
	std::vector<int32_t> cid(n);
	std::vector<double> r(3 * n), v(3 * n);
	int st = mdgpu_get_particles(ctx, n, id.data(), cid.data(), r.data(), v.data(), nullptr);
	if (st) return st;
	const std::string head = mdgpu::checkpoint_header(c, n, current_time, temperature, epsilon_rf);
	// molecule lines formatted in parallel ranges, written in order
	const unsigned parts = mdgpu::worker_count(n);
	std::vector<std::string> body(parts);
	mdgpu::parallel_ranges(n, parts, [&](unsigned k, int64_t lo, int64_t hi) {
		std::string& out = body[k];
		out.reserve((size_t) (hi - lo) * (size_t) (40 + 8 * (digits + 7)));
		char b[512];
		for (int64_t i = lo; i < hi; i++) {
			const int len = snprintf(b, sizeof(b), "%llu\t%d\t%.*g %.*g %.*g\t%.*g %.*g %.*g\t1 0 0 0\t0 0 0\t\n",
			                         (unsigned long long) id[i], cid[i] + 1, digits, r[3 * i], digits, r[3 * i + 1],
			                         digits, r[3 * i + 2], digits, v[3 * i], digits, v[3 * i + 1], digits, v[3 * i + 2]);
			out.append(b, (size_t) len);
		}
	});
	FILE* f = fopen(path, "wb");
	if (!f) return mdgpu::io_fail(c, MDGPU_ERR_ARG, std::string("cannot open ") + path + ": " + strerror(errno));
	bool ok = fwrite(head.data(), 1, head.size(), f) == head.size();
	for (const std::string& s : body) ok = ok && fwrite(s.data(), 1, s.size(), f) == s.size();
	ok = (fclose(f) == 0) && ok;
	if (!ok) return mdgpu::io_fail(c, MDGPU_ERR_ARG, std::string("write failed: ") + path);
	return MDGPU_OK;
}

int mdgpu_read_phase_space(mdgpu_ctx* ctx, const char* path, double* current_time, double* temperature) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (!path) return mdgpu::io_fail(c, MDGPU_ERR_ARG, "path is required");
	FILE* f = fopen(path, "rb");
	if (!f) return mdgpu::io_fail(c, MDGPU_ERR_ARG, std::string("cannot open ") + path + ": " + strerror(errno));
	std::string text;
	{
		fseek(f, 0, SEEK_END);
		const long size = ftell(f);
		fseek(f, 0, SEEK_SET);
		text.resize(size > 0 ? (size_t) size : 0);
		const size_t got = size > 0 ? fread(&text[0], 1, (size_t) size, f) : 0;
		fclose(f);
		if (got != text.size()) return mdgpu::io_fail(c, MDGPU_ERR_ARG, std::string("read failed: ") + path);
	}
	// comment lines (starting with '#') are blanked, as the reference's header reader skips them
	for (size_t i = 0; i < text.size();) {
		size_t j = i;
		while (j < text.size() && (text[j] == ' ' || text[j] == '\t')) j++;
		size_t e = text.find('\n', i);
		if (e == std::string::npos) e = text.size();
		if (j < text.size() && text[j] == '#') std::fill(text.begin() + (long) i, text.begin() + (long) e, ' ');
		i = e + 1;
	}
	mdgpu::Cursor cur{text.data(), text.data() + text.size()};
	std::string tok;
	auto bad = [&](const std::string& why) { return mdgpu::io_fail(c, MDGPU_ERR_ARG, std::string(path) + ": " + why); };
	// InputOldstyle::readPhaseSpaceHeader (io/InputOldstyle.cpp:35-259)
	if (!cur.token(tok) || !(tok == "mardyn" || tok == "MOLDY" || tok == "ls1r1" || tok == "mrdyn" ||
	                         tok == "MDProject" || tok == "Mardyn" || tok == "MARDYN"))
		return bad("not a valid OldStyle input file");
	if (!cur.token(tok) || tok != "trunk") return bad("wrong input file specifier");
	if (!cur.token(tok)) return bad("missing version");
	double t_cur = 0.0, t_target = 1.0;
	double length[3] = {0, 0, 0};
	bool have_length = false, have_components = false;
	while (!have_components) {
		if (!cur.token(tok)) return bad("header ends before NumberOfComponents");
		double x;
		if (tok == "currentTime" || tok == "t") {
			if (!cur.number(t_cur)) return bad("bad currentTime");
		} else if (tok == "Temperature" || tok == "T") {
			if (!cur.number(t_target)) return bad("bad Temperature");
		} else if (tok == "ThermostatTemperature" || tok == "ThT" || tok == "h") {
			if (!cur.number(x) || !cur.number(x)) return bad("bad ThermostatTemperature");
		} else if (tok == "ComponentThermostat" || tok == "CT" || tok == "o") {
			if (!cur.number(x) || !cur.number(x)) return bad("bad ComponentThermostat");
		} else if (tok == "Undirected" || tok == "U") {
			if (!cur.number(x)) return bad("bad Undirected");
		} else if (tok == "Length" || tok == "L") {
			if (!cur.number(length[0]) || !cur.number(length[1]) || !cur.number(length[2])) return bad("bad Length");
			have_length = true;
		} else if (tok == "HeatCapacity" || tok == "cv" || tok == "I") {
			if (!cur.number(x) || !cur.number(x) || !cur.number(x)) return bad("bad HeatCapacity");
		} else if (tok == "AssignCoset" || tok == "S") {
			if (!cur.number(x) || !cur.number(x)) return bad("bad AssignCoset");
		} else if (tok == "Accelerate" || tok == "A") {
			for (int k = 0; k < 8; k++)
				if (!cur.number(x)) return bad("bad Accelerate");
		} else if (tok == "NumberOfComponents" || tok == "C") {
			double ncd;
			if (!cur.number(ncd)) return bad("bad NumberOfComponents");
			const int nc = (int) ncd;
			if (nc != c->sp.n) return bad("the file has " + std::to_string(nc) + " components, the context " +
			                              std::to_string(c->sp.n));
			for (int i = 0; i < nc; i++) {
				double cnt[5];
				for (double& k : cnt)
					if (!cur.number(k)) return bad("bad component site counts");
				if (cnt[0] != 1 || cnt[1] != 0 || cnt[2] != 0 || cnt[3] != 0 || cnt[4] != 0)
					return bad("only single-site LJ components are supported");
				double s[8];
				for (double& k : s)
					if (!cur.number(k)) return bad("bad LJ centre");
				if (s[0] != 0 || s[1] != 0 || s[2] != 0) return bad("the LJ centre must sit at the molecule origin");
				if (!mdgpu::close_to(s[3], c->sp.mass[i]) || !mdgpu::close_to(s[4], c->eps[i]) ||
				    !mdgpu::close_to(s[5], c->sigma[i]))
					return bad("component " + std::to_string(i + 1) + " differs from the context's");
				double ipa[3];
				for (double& k : ipa)
					if (!cur.number(k)) return bad("bad moments of inertia");
			}
			for (int k = 0; k < nc * (nc - 1); k++)
				if (!cur.number(x)) return bad("bad mixing coefficients");
			if (!cur.number(x)) return bad("bad epsilonRF");
			have_components = true;
		} else {
			return bad("invalid header token '" + tok + "'");
		}
	}
	if (have_length)
		for (int d = 0; d < 3; d++)
			if (!mdgpu::close_to(length[d], c->g.L[d])) return bad("the box lengths differ from the context's");
	// InputOldstyle::readPhaseSpace (io/InputOldstyle.cpp:261-392)
	double nd;
	if (!cur.token(tok) || !(tok == "NumberOfMolecules" || tok == "N") || !cur.number(nd))
		return bad("expected NumberOfMolecules");
	const int64_t n = (int64_t) nd;
	if (n < 1) return bad("no molecules");
	enum { kICRVQD, kIRV, kICRV, kICRVFQDM } fmt = kICRVQD;
	{
		mdgpu::Cursor save = cur;
		if (cur.token(tok) && (tok == "MoleculeFormat" || tok == "M")) {
			if (!cur.token(tok)) return bad("missing molecule format");
			if (tok == "ICRVQD")
				fmt = kICRVQD;
			else if (tok == "ICRVFQDM")
				fmt = kICRVFQDM;
			else if (tok == "ICRV")
				fmt = kICRV;
			else if (tok == "IRV")
				fmt = kIRV;
			else
				return bad("unknown molecule format '" + tok + "'");
		} else {
			cur = save;
		}
	}
	const int fields = fmt == kICRVQD ? 15 : fmt == kICRVFQDM ? 21 : fmt == kICRV ? 8 : 7;
	// molecule records: split the rest at line starts into ranges parsed in parallel
	const char* body = cur.p;
	const char* end = cur.end;
	std::vector<const char*> lines;
	lines.reserve((size_t) n + 1);
	for (const char* q = body; q < end;) {
		while (q < end && (*q == ' ' || *q == '\t' || *q == '\r' || *q == '\n')) q++;
		if (q >= end) break;
		lines.push_back(q);
		const void* nl = memchr(q, '\n', (size_t) (end - q));
		q = nl ? (const char*) nl + 1 : end;
	}
	if ((int64_t) lines.size() < n) return bad("fewer molecule lines than NumberOfMolecules");
	std::vector<uint64_t> id((size_t) n);
	std::vector<int32_t> cid((size_t) n);
	std::vector<double> r(3 * (size_t) n), v(3 * (size_t) n), F;
	if (fmt == kICRVFQDM) F.resize(3 * (size_t) n);
	const unsigned parts = mdgpu::worker_count(n);
	std::vector<int64_t> first_bad(parts, -1);
	const int nspec = c->sp.n;
	mdgpu::parallel_ranges(n, parts, [&](unsigned k, int64_t lo, int64_t hi) {
		double vals[21];
		for (int64_t i = lo; i < hi; i++) {
			const char* q = lines[(size_t) i];
			const char* stop = (size_t) i + 1 < lines.size() ? lines[(size_t) i + 1] : end;
			bool ok = true;
			for (int f = 0; f < fields && ok; f++) {
				char* e = nullptr;
				vals[f] = strtod(q, &e);
				ok = e != q && e <= stop;
				q = e;
			}
			int32_t ci = 0;
			int o = 1;
			if (fmt != kIRV) {
				ci = (int32_t) vals[1] - 1;
				o = 2;
			}
			if (!ok || ci < 0 || ci >= nspec || vals[0] < 0) {
				if (first_bad[k] < 0) first_bad[k] = i;
				continue;
			}
			id[(size_t) i] = (uint64_t) vals[0];
			cid[(size_t) i] = ci;
			for (int d = 0; d < 3; d++) {
				r[3 * (size_t) i + d] = vals[o + d];
				v[3 * (size_t) i + d] = vals[o + 3 + d];
			}
			if (fmt == kICRVFQDM)
				for (int d = 0; d < 3; d++) F[3 * (size_t) i + d] = vals[o + 6 + d];
		}
	});
	for (int64_t b : first_bad)
		if (b >= 0) return bad("malformed molecule record " + std::to_string(b + 1));
	int st = mdgpu_set_particles(ctx, n, id.data(), cid.data(), r.data(), v.data(), F.empty() ? nullptr : F.data());
	if (st) return st;
	if (current_time) *current_time = t_cur;
	if (temperature) *temperature = t_target;
	return MDGPU_OK;
}
