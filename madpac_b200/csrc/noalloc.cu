// Allocation-free force evaluation: mdgpu_forces_noalloc.
//
// Who needs it: callers that cannot call cudaMalloc while they run this code. Examples are hosts
// that own all device memory through their own pool allocator (a foreign cudaMalloc would bypass
// their accounting or fail once the pool has reserved the device), and latency-bound loops that
// must not block on the driver's allocator. They pass device buffers they already own for the
// inputs and outputs; every intermediate buffer of the binning and the pair traversal (sorted
// copies of the molecules, cell counts and offsets, reduction partials, status word, parameter
// table) comes from one file-scope device array, g_scratch, sized for at most
// kNoAllocMaxMolecules molecules and kNoAllocMaxCells cells.
//
// The call is synchronous: it uploads its parameter table from host memory, waits for its stream
// and returns Upot, the virial and the status on the host.
//
// Consequences of a static scratch array:
//  * every GPU that loads the library holds g_scratch (about 7.5 MB) until the process exits;
//  * all calls on one device share it, and it keeps the contents of the last call: each call
//    clears what must start at zero (status word, cell counts) before using it;
//  * calls that overlap on the GPU (other host threads, or several streams in flight) race on
//    g_scratch and corrupt each other's results -- serialise them;
//  * the first call on a device looks up g_scratch's device address (cudaGetSymbolAddress, with
//    that device current) and keeps it for the rest of the process; make that first call before
//    any stream capture begins, and do not use the library across a cudaDeviceReset of that
//    device (the module, and with it g_scratch, is loaded again at another address).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "md_internal.h"

namespace mdgpu {
namespace {

constexpr int64_t kNoAllocMaxMolecules = 32768;
constexpr int64_t kNoAllocMaxCells = 32768;

constexpr size_t na_align(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of every buffer inside g_scratch.
struct NaLayout {
	size_t p, q, cell, rank, perm, count, start, scan, partials, scalars, status, params, total;
};

constexpr size_t kParticleBytes = na_align((9 * sizeof(double) + sizeof(uint64_t) + 2 * sizeof(int32_t)) *
                                           kNoAllocMaxMolecules);
constexpr int64_t kPartialBlocks = kNoAllocMaxCells + kNoAllocMaxMolecules / kReduceBlock + 1024 + 1;

constexpr NaLayout na_layout() {
	NaLayout L{};
	size_t o = 0;
	L.p = o;
	o += kParticleBytes;
	L.q = o;
	o += kParticleBytes;
	L.cell = o;
	o += na_align(sizeof(int32_t) * kNoAllocMaxMolecules);
	L.rank = o;
	o += na_align(sizeof(int32_t) * kNoAllocMaxMolecules);
	L.perm = o;
	o += na_align(sizeof(int32_t) * kNoAllocMaxMolecules);
	L.count = o;
	o += na_align(sizeof(int32_t) * kNoAllocMaxCells);
	L.start = o;
	o += na_align(sizeof(int32_t) * (kNoAllocMaxCells + 1));
	L.scan = o;
	o += na_align(sizeof(int32_t) * (kNoAllocMaxCells / 1024 + 2));
	L.partials = o;
	o += na_align(sizeof(double) * 4 * kPartialBlocks);
	L.scalars = o;
	o += na_align(sizeof(double) * 64);
	L.status = o;
	o += na_align(sizeof(int));
	L.params = o;
	o += na_align(sizeof(PairParams));
	L.total = o;
	return L;
}

constexpr NaLayout kNaLayout = na_layout();

static __device__ __align__(256) unsigned char g_scratch[kNaLayout.total];

std::mutex g_mutex;
unsigned char* g_addr[kMaxDevices] = {};

// Particle arrays carved out of one kParticleBytes region.
Particles carve(unsigned char* base) {
	Particles p{};
	const int64_t n = kNoAllocMaxMolecules;
	double* d = reinterpret_cast<double*>(base);
	p.rx = d;
	p.ry = d + n;
	p.rz = d + 2 * n;
	p.vx = d + 3 * n;
	p.vy = d + 4 * n;
	p.vz = d + 5 * n;
	p.fx = d + 6 * n;
	p.fy = d + 7 * n;
	p.fz = d + 8 * n;
	p.id = reinterpret_cast<uint64_t*>(d + 9 * n);
	p.cid = reinterpret_cast<int32_t*>(p.id + n);
	p.uidx = p.cid + n;
	return p;
}

// caller's (n, 3) positions and component ids -> sorted-order arrays (initially caller order)
__global__ void k_na_load(int64_t n, const double* __restrict__ r, const int32_t* __restrict__ cid, int ns,
                          Particles p, int* status) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	p.rx[s] = r[3 * s];
	p.ry[s] = r[3 * s + 1];
	p.rz[s] = r[3 * s + 2];
	p.vx[s] = p.vy[s] = p.vz[s] = 0.0;
	p.fx[s] = p.fy[s] = p.fz[s] = 0.0;
	int t = cid[s];
	if (t < 0 || t >= ns) {
		atomicOr(status, kStatusCapacity);
		t = 0;
	}
	p.cid[s] = t;
	p.id[s] = (uint64_t) s;
	p.uidx[s] = (int32_t) s;
}

// sorted-order forces -> caller's (n, 3) array
__global__ void k_na_store(int64_t n, Particles p, double* __restrict__ F) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const int64_t u = p.uidx[s];
	F[3 * u] = p.fx[s];
	F[3 * u + 1] = p.fy[s];
	F[3 * u + 2] = p.fz[s];
}

// Restores the calling thread's current device when the entry point returns.
struct DeviceGuard {
	int dev;
	explicit DeviceGuard(int d) : dev(d) {}
	~DeviceGuard() {
		if (dev >= 0) cudaSetDevice(dev);
	}
};

int na_fail(char* errbuf, int errlen, int code, const char* msg) {
	if (errbuf && errlen > 0) snprintf(errbuf, (size_t) errlen, "%s", msg);
	return code;
}

}  // namespace
}  // namespace mdgpu

using namespace mdgpu;

extern "C" int mdgpu_forces_noalloc(int device, void* stream, int64_t n, const double* d_r, const int32_t* d_cid,
                                    const double length[3], double cutoff, double lj_cutoff, int ncomp,
                                    const mdgpu_component* comps, const double* mix, int precision, double* d_F,
                                    double* upot, double* virial, char* errbuf, int errlen) {
	if (errbuf && errlen > 0) errbuf[0] = '\0';
	if (n < 1 || n > kNoAllocMaxMolecules)
		return na_fail(errbuf, errlen, MDGPU_ERR_CAPACITY,
		               "mdgpu_forces_noalloc: n must be in 1..32768 (the size of its static scratch array)");
	if (!d_r || !d_cid || !d_F || !length || !comps) return na_fail(errbuf, errlen, MDGPU_ERR_ARG, "null argument");
	if (ncomp < 1 || ncomp > kMaxSpecies) return na_fail(errbuf, errlen, MDGPU_ERR_ARG, "ncomp must be in 1..8");
	if (ncomp > 1 && !mix) return na_fail(errbuf, errlen, MDGPU_ERR_ARG, "mixing coefficients required");
	if (!(cutoff > 0)) return na_fail(errbuf, errlen, MDGPU_ERR_ARG, "cutoff must be positive");
	if (!(lj_cutoff >= 0))
		return na_fail(errbuf, errlen, MDGPU_ERR_ARG, "lj_cutoff must be 0 (= cutoff) or positive");
	if (precision != MDGPU_FP64 && precision != MDGPU_MIXED)
		return na_fail(errbuf, errlen, MDGPU_ERR_ARG, "unknown precision mode");
	if (device < 0 || device >= kMaxDevices) return na_fail(errbuf, errlen, MDGPU_ERR_ARG, "device out of range");

	Context c;
	c.device = device;
	c.stream = reinterpret_cast<cudaStream_t>(stream);
	c.precision = precision;
	c.rc = cutoff;
	c.rc_lj = lj_cutoff == 0.0 ? cutoff : lj_cutoff;
	// cell grid of the bounding box [0, L), as LinkedCells' constructor (LinkedCells.cpp:54-71)
	int64_t ncells = 1;
	for (int d = 0; d < 3; d++) {
		if (!(length[d] > 0)) return na_fail(errbuf, errlen, MDGPU_ERR_ARG, "box lengths must be positive");
		int w = (int) std::floor((length[d] - 0.0) / cutoff * 1.0);
		if (w < 2) return na_fail(errbuf, errlen, MDGPU_ERR_BOX_TOO_SMALL, "the box must hold 2 cells per dimension");
		c.g.nc[d] = w;
		c.g.L[d] = length[d];
		c.g.cell_length[d] = (length[d] - 0.0) / w;
		c.g.halo_min[d] = 0.0 - 1 * c.g.cell_length[d];
		ncells *= w;
	}
	if (ncells > kNoAllocMaxCells)
		return na_fail(errbuf, errlen, MDGPU_ERR_CAPACITY,
		               "mdgpu_forces_noalloc: the box has more than 32768 cells (the size of its static scratch array)");
	c.g.ncells = ncells;
	// Comp2Param stream entries (Comp2Param.cpp:28-115; shift6 of Component::addLJcenter)
	PairParams hp{};
	hp.ns = ncomp;
	hp.rc2 = c.rc * c.rc;
	hp.rclj2 = c.rc_lj * c.rc_lj;
	c.sp.n = ncomp;
	int mixpos = 0;
	for (int i = 0; i < ncomp; i++) {
		const mdgpu_component& a = comps[i];
		if (!(a.mass > 0)) return na_fail(errbuf, errlen, MDGPU_ERR_ARG, "component masses must be positive");
		c.sp.mass[i] = a.mass;
		double shift6i = 0.0;
		if (a.do_shift) {
			double sigperrc2 = a.sigma * a.sigma / (c.rc_lj * c.rc_lj);
			double sigperrc6 = sigperrc2 * sigperrc2 * sigperrc2;
			shift6i = 24.0 * a.eps * (sigperrc6 - sigperrc6 * sigperrc6);
		}
		double sg = .5 * (a.sigma + a.sigma);
		hp.eps24[i * ncomp + i] = 24. * std::sqrt(a.eps * a.eps);
		hp.sig2[i * ncomp + i] = sg * sg;
		hp.shift6[i * ncomp + i] = shift6i;
		for (int j = i + 1; j < ncomp; j++) {
			const mdgpu_component& b = comps[j];
			double xi = mix[mixpos++], eta = mix[mixpos++];
			for (int dir = 0; dir < 2; dir++) {
				double ea = dir ? b.eps : a.eps, eb = dir ? a.eps : b.eps;
				double sa = dir ? b.sigma : a.sigma, sb = dir ? a.sigma : b.sigma;
				double epsilon24 = 24. * xi * std::sqrt(ea * eb);
				double sigma2 = eta * .5 * (sa + sb);
				sigma2 *= sigma2;
				double sigperrc2 = sigma2 / (c.rc_lj * c.rc_lj);
				double sigperrc6 = sigperrc2 * sigperrc2 * sigperrc2;
				int k = dir ? j * ncomp + i : i * ncomp + j;
				hp.eps24[k] = epsilon24;
				hp.sig2[k] = sigma2;
				hp.shift6[k] = epsilon24 * (sigperrc6 - sigperrc6 * sigperrc6);
			}
		}
	}
	for (int k = 0; k < kMaxSpecies * kMaxSpecies; k++) {
		c.sp.eps24[k] = hp.eps24[k];
		c.sp.sig2[k] = hp.sig2[k];
		c.sp.shift6[k] = hp.shift6[k];
	}

	// the caller's current device is put back on every return below
	int prev_device = -1;
	cudaError_t e = cudaGetDevice(&prev_device);
	if (e != cudaSuccess) return na_fail(errbuf, errlen, MDGPU_ERR_CUDA, cudaGetErrorString(e));
	DeviceGuard guard(prev_device);
	e = cudaSetDevice(device);
	if (e != cudaSuccess) return na_fail(errbuf, errlen, MDGPU_ERR_CUDA, cudaGetErrorString(e));
	unsigned char* base = nullptr;
	{
		std::lock_guard<std::mutex> lock(g_mutex);
		if (!g_addr[device]) {
			void* ptr = nullptr;
			e = cudaGetSymbolAddress(&ptr, g_scratch);
			if (e != cudaSuccess) return na_fail(errbuf, errlen, MDGPU_ERR_CUDA, cudaGetErrorString(e));
			g_addr[device] = static_cast<unsigned char*>(ptr);
		}
		base = g_addr[device];
	}
	const NaLayout& L = kNaLayout;
	c.n = n;
	c.cap = n;
	c.p = carve(base + L.p);
	c.q = carve(base + L.q);
	c.cell = reinterpret_cast<int32_t*>(base + L.cell);
	c.rank = reinterpret_cast<int32_t*>(base + L.rank);
	c.perm = reinterpret_cast<int32_t*>(base + L.perm);
	c.cell_count = reinterpret_cast<int32_t*>(base + L.count);
	c.cell_start = reinterpret_cast<int32_t*>(base + L.start);
	c.scan_tmp = reinterpret_cast<int32_t*>(base + L.scan);
	c.scan_blocks = (ncells + 1023) / 1024;
	c.partials = reinterpret_cast<double*>(base + L.partials);
	c.partial_cap = kPartialBlocks;
	c.scalars = reinterpret_cast<double*>(base + L.scalars);
	c.status = reinterpret_cast<int*>(base + L.status);
	c.d_pp = reinterpret_cast<PairParams*>(base + L.params);
	c.pair_kernel = 0;

	// the shared array keeps the previous call's contents: clear the status word (the binning
	// clears the cell counts itself) and upload this call's parameter table
	e = cudaMemsetAsync(c.status, 0, sizeof(int), c.stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(c.d_pp, &hp, sizeof(PairParams), cudaMemcpyHostToDevice, c.stream);
	if (e == cudaSuccess) {
		k_na_load<<<(unsigned) ((n + 255) / 256), 256, 0, c.stream>>>(n, d_r, d_cid, ncomp, c.p, c.status);
		e = cudaGetLastError();
	}
	if (e == cudaSuccess) e = launch_bin(&c, false);
	if (e == cudaSuccess) e = launch_pairs(&c);
	if (e == cudaSuccess) {
		k_na_store<<<(unsigned) ((n + 255) / 256), 256, 0, c.stream>>>(n, c.p, d_F);
		e = cudaGetLastError();
	}
	double sc[3] = {0, 0, 0};
	int st = 0;
	if (e == cudaSuccess) e = cudaMemcpyAsync(sc, c.scalars, sizeof(sc), cudaMemcpyDeviceToHost, c.stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(&st, c.status, sizeof(int), cudaMemcpyDeviceToHost, c.stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
	if (e != cudaSuccess) return na_fail(errbuf, errlen, MDGPU_ERR_CUDA, cudaGetErrorString(e));
	if (st & kStatusOutsideHalo) return na_fail(errbuf, errlen, MDGPU_ERR_OUTSIDE_HALO, "a molecule is outside the box");
	if (st & kStatusSamePosition)
		return na_fail(errbuf, errlen, MDGPU_ERR_SAME_POSITION, "two molecules have the same position");
	if (st & kStatusNonFinite) return na_fail(errbuf, errlen, MDGPU_ERR_NONFINITE, "non-finite force");
	if (st & kStatusCapacity) return na_fail(errbuf, errlen, MDGPU_ERR_ARG, "component id out of range");
	// ParticlePairs2PotForceAdapter::finish: each pair was evaluated from both sides
	if (upot) *upot = sc[0] * 0.5 / 6.;
	if (virial) *virial = sc[1] * 0.5;
	return MDGPU_OK;
}
