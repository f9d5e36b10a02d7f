// C ABI of the LJ hot path (include/mdgpu.h): context set-up, particle I/O in caller order,
// the step sequence and device-side timing.
#include <cuda_runtime.h>

#include <mutex>

#include <utility>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "md_internal.h"

using mdgpu::Context;

namespace mdgpu {
namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(int64_t n) { return (unsigned) ((n + kThreads - 1) / kThreads); }

// caller order (AoS, n x 3) -> sorted SoA through uidx
__global__ void k_load_aos(int64_t n, const double* __restrict__ aos, const int32_t* __restrict__ uidx,
                           double* __restrict__ x, double* __restrict__ y, double* __restrict__ z) {
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	int64_t u = uidx ? uidx[s] : s;
	x[s] = aos[3 * u + 0];
	y[s] = aos[3 * u + 1];
	z[s] = aos[3 * u + 2];
}

// sorted SoA -> caller order (AoS)
__global__ void k_store_aos(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const int32_t* __restrict__ uidx, double* __restrict__ aos) {
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	int64_t u = uidx[s];
	aos[3 * u + 0] = x[s];
	aos[3 * u + 1] = y[s];
	aos[3 * u + 2] = z[s];
}

// positions -> caller order with the periodic wrap r<0 -> r+L, r>=L -> r-L
__global__ void k_store_pos(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const int32_t* __restrict__ uidx, Grid g,
                            double* __restrict__ aos) {
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	int64_t u = uidx[s];
	const double r[3] = {x[s], y[s], z[s]};
	for (int d = 0; d < 3; d++) {
		double w = r[d];
		if (w < 0.0)
			w = __dadd_rn(w, g.L[d]);
		else if (w >= g.L[d])
			w = __dsub_rn(w, g.L[d]);
		aos[3 * u + d] = w;
	}
}

template <typename T>
__global__ void k_store_scalar(int64_t n, const T* __restrict__ x, const int32_t* __restrict__ uidx, T* __restrict__ out) {
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n) out[uidx[s]] = x[s];
}

// inner cell -> reference halo-inclusive cell index, caller order
__global__ void k_store_refcell(int64_t n, const int32_t* __restrict__ cell, const int32_t* __restrict__ uidx, Grid g,
                                int64_t* __restrict__ out) {
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	int c = cell[s];
	int ix = c % g.nc[0], iy = (c / g.nc[0]) % g.nc[1], iz = c / (g.nc[0] * g.nc[1]);
	int64_t cx = g.nc[0] + 2, cy = g.nc[1] + 2;
	out[uidx[s]] = ((int64_t) (iz + 1) * cy + (iy + 1)) * cx + (ix + 1);
}

__global__ void k_set_int(int* p, int v) { *p = v; }

__global__ void k_iota(int64_t n, int32_t* __restrict__ a) {
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n) a[s] = (int32_t) s;
}

int fail(Context* c, int code, const std::string& msg) {
	c->err = msg;
	return code;
}

int cuda_fail(Context* c, cudaError_t e, const char* where) {
	c->err = std::string(where) + ": " + cudaGetErrorString(e);
	return MDGPU_ERR_CUDA;
}

#define MD_CUDA(call)                                         \
	do {                                                      \
		cudaError_t e_ = (call);                              \
		if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
	} while (0)

// Reads and clears the device status word (synchronises the stream).
int check_status(Context* c) {
	MD_CUDA(cudaMemcpyAsync(c->h_status, c->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
	MD_CUDA(cudaStreamSynchronize(c->stream));
	int st = *c->h_status;
	if (st == 0) return MDGPU_OK;
	MD_CUDA(cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
	if (st & kStatusOutsideHalo)
		return fail(c, MDGPU_ERR_OUTSIDE_HALO, "a molecule is outside the halo box (moved more than one cell in a step)");
	if (st & kStatusSamePosition) return fail(c, MDGPU_ERR_SAME_POSITION, "two molecules have the same position");
	if (st & kStatusNonFinite) return fail(c, MDGPU_ERR_NONFINITE, "non-finite force or velocity");
	if (st & kStatusTimeout) {
		// the cooperative rebuild's barrier words may be left mid-count: start them again
		if (c->bar) MD_CUDA(cudaMemsetAsync(c->bar, 0, sizeof(unsigned) * 4, c->stream));
		// ... and its counts and look-back words, which it clears only when it runs to the end
		if (c->rb_count) MD_CUDA(cudaMemsetAsync(c->rb_count, 0, sizeof(int32_t) * c->g.ncells, c->stream));
		if (c->rb_look) MD_CUDA(cudaMemsetAsync(c->rb_look, 0, sizeof(unsigned long long) * c->rb_look_cap, c->stream));
		c->lists_valid = false;
		return fail(c, MDGPU_ERR_TIMEOUT, "a bounded device wait gave up");
	}
	if (st & kStatusCapacity) return fail(c, MDGPU_ERR_CAPACITY, "a device buffer is too small for the workload");
	if (st & kStatusRange)
		return fail(c, MDGPU_ERR_CAPACITY, "a per-cell fixed-point sum left its range (|sum| >= 2^23)");
	return fail(c, MDGPU_ERR_CUDA, "unknown device status");
}

void free_particles(Particles& p) {
	cudaFree(p.rx);
	cudaFree(p.ry);
	cudaFree(p.rz);
	cudaFree(p.vx);
	cudaFree(p.vy);
	cudaFree(p.vz);
	cudaFree(p.fx);
	cudaFree(p.fy);
	cudaFree(p.fz);
	cudaFree(p.id);
	cudaFree(p.cid);
	cudaFree(p.uidx);
	p = Particles{};
}

cudaError_t alloc_particles(Particles& p, int64_t n) {
	double** d[] = {&p.rx, &p.ry, &p.rz, &p.vx, &p.vy, &p.vz, &p.fx, &p.fy, &p.fz};
	for (double** a : d) {
		cudaError_t e = cudaMalloc(a, sizeof(double) * n);
		if (e != cudaSuccess) return e;
	}
	cudaError_t e = cudaMalloc(&p.id, sizeof(uint64_t) * n);
	if (e == cudaSuccess) e = cudaMalloc(&p.cid, sizeof(int32_t) * n);
	if (e == cudaSuccess) e = cudaMalloc(&p.uidx, sizeof(int32_t) * n);
	return e;
}

// Staging buffer for AoS transfers (n x 3 doubles), reused between calls.
struct Staging {
	void* ptr = nullptr;
	size_t bytes = 0;
};

cudaError_t staging(Context* c, Staging& st, size_t bytes, void** out) {
	if (st.bytes < bytes) {
		cudaFree(st.ptr);
		st.ptr = nullptr;
		cudaError_t e = cudaMalloc(&st.ptr, bytes);
		if (e != cudaSuccess) {
			st.bytes = 0;
			return e;
		}
		st.bytes = bytes;
	}
	*out = st.ptr;
	return cudaSuccess;
}

struct Extra {
	Staging stage;
	std::vector<int64_t> species_count;
	// timing records
	struct Rec {
		int group;
		cudaEvent_t a, b;
	};
	std::vector<Rec> recs;
	std::vector<cudaEvent_t> pool;
	cudaEvent_t open_a[3] = {nullptr, nullptr, nullptr};
};

Extra* extra(Context* c);

}  // namespace

void count_launches(Context* c, int launches) { c->prof_count[3] += launches; }

int check_device_status(Context* c) { return check_status(c); }

int set_error(Context* c, int code, const std::string& msg) { return fail(c, code, msg); }

int set_cuda_error(Context* c, cudaError_t e, const char* where) { return cuda_fail(c, e, where); }

void prof_begin(Context* c, int group) {
	if (!c->profiling) return;
	Extra* x = extra(c);
	cudaEvent_t a;
	if (!x->pool.empty()) {
		a = x->pool.back();
		x->pool.pop_back();
	} else {
		cudaEventCreate(&a);
	}
	cudaEventRecord(a, c->stream);
	x->open_a[group] = a;
}

void prof_end(Context* c, int group, int launches) {
	c->prof_count[group] += launches;
	c->prof_count[3] += launches;
	if (!c->profiling) return;
	Extra* x = extra(c);
	cudaEvent_t b;
	if (!x->pool.empty()) {
		b = x->pool.back();
		x->pool.pop_back();
	} else {
		cudaEventCreate(&b);
	}
	cudaEventRecord(b, c->stream);
	x->recs.push_back({group, x->open_a[group], b});
}

}  // namespace mdgpu

// The Extra block lives right after the context in one allocation.
struct mdgpu_ctx_full {
	mdgpu_ctx pub;
	mdgpu::Extra x;
};

namespace mdgpu {
namespace {
Extra* extra(Context* c) { return &reinterpret_cast<mdgpu_ctx_full*>(reinterpret_cast<mdgpu_ctx*>(c))->x; }
}  // namespace
}  // namespace mdgpu

namespace mdgpu {

int setup_grid(const double length[3], double cutoff, double cells_in_cutoff, Grid& g, std::string& err) {
	// LinkedCells geometry for the bounding box [0, L) (LinkedCells.cpp:54-71)
	int64_t ncells = 1;
	for (int d = 0; d < 3; d++) {
		if (!(length[d] > 0)) {
			err = "box lengths must be positive";
			return MDGPU_ERR_ARG;
		}
		double bbmin = 0.0, bbmax = length[d];
		int w = (int) std::floor((bbmax - bbmin) / cutoff * cells_in_cutoff);
		if (w == 0) w = 1;
		if (w < 2) {
			err = "the box must hold at least 2 cells of edge >= cutoff in every dimension";
			return MDGPU_ERR_BOX_TOO_SMALL;
		}
		g.nc[d] = w;
		g.L[d] = length[d];
		g.cell_length[d] = (bbmax - bbmin) / w;
		double halo_len = 1 * g.cell_length[d];
		g.halo_min[d] = bbmin - halo_len;
		ncells *= w;
	}
	if (ncells > (int64_t) 0x7fffffff) {
		err = "too many cells";
		return MDGPU_ERR_CAPACITY;
	}
	g.ncells = ncells;
	return MDGPU_OK;
}

// The Verlet-skin grid: cells of edge >= cutoff + skin, so that every molecule that can come within
// the cutoff before the next build is in the 27 cells around; in a dilute liquid larger, so that a
// cell holds about kSkinCellOcc molecules at the density around a typical molecule and a 2x2x2
// brick fills the eight warps of its CTA; an even count per dimension where it is 5 or more.
constexpr double kSkinCellOcc = 28.0;
int skin_grid(const Context* c, double skin, Grid& gs, std::string& err) {
	double edge = c->rc + skin;
	if (c->rho_typ > 0.0) edge = std::max(edge, std::cbrt(kSkinCellOcc / c->rho_typ));
	const double length[3] = {c->g.L[0], c->g.L[1], c->g.L[2]};
	int st = setup_grid(length, edge, 1.0, gs, err);
	// larger cells only where every dimension keeps 3 or more: with 2, one brick would hold the
	// whole box and stage it eight times over
	if (edge > c->rc + skin && (st || gs.nc[0] < 3 || gs.nc[1] < 3 || gs.nc[2] < 3))
		st = setup_grid(length, c->rc + skin, 1.0, gs, err);
	if (st) return st;
	even_grid(gs);
	return MDGPU_OK;
}

void even_grid(Grid& g) {
	// 2x2x2-cell bricks tile an even number of cells exactly; with an odd count the last brick of
	// a row owns one cell and leaves most of its CTA idle. Larger cells keep every pair within
	// the radius inside the 27 cells around a molecule. Three cells stay three (two would make
	// one brick of the whole box, staged eight times over).
	int64_t ncells = 1;
	for (int d = 0; d < 3; d++) {
		if (g.nc[d] >= 5 && (g.nc[d] & 1)) {
			g.nc[d] -= 1;
			g.cell_length[d] = g.L[d] / g.nc[d];
			g.halo_min[d] = -g.cell_length[d];
		}
		ncells *= g.nc[d];
	}
	g.ncells = ncells;
}

int setup_species(int ncomp, const mdgpu_component* comps, const double* mix, double rcLJ, Species& sp,
                  std::string& err) {
	// Comp2Param stream entries (Comp2Param.cpp:28-115; shift6 of Component::addLJcenter,
	// Component.cpp:47-55), one LJ centre per component
	sp = Species{};
	sp.n = ncomp;
	int mixpos = 0;
	for (int i = 0; i < ncomp; i++) {
		const mdgpu_component& a = comps[i];
		if (!(a.mass > 0)) {
			err = "component masses must be positive";
			return MDGPU_ERR_ARG;
		}
		sp.mass[i] = a.mass;
		double shift6i = 0.0;
		if (a.do_shift) {
			double sigperrc2 = a.sigma * a.sigma / (rcLJ * rcLJ);
			double sigperrc6 = sigperrc2 * sigperrc2 * sigperrc2;
			shift6i = 24.0 * a.eps * (sigperrc6 - sigperrc6 * sigperrc6);
		}
		double sg = .5 * (a.sigma + a.sigma);
		sp.eps24[i * ncomp + i] = 24. * std::sqrt(a.eps * a.eps);
		sp.sig2[i * ncomp + i] = sg * sg;
		sp.shift6[i * ncomp + i] = shift6i;
		for (int j = i + 1; j < ncomp; j++) {
			const mdgpu_component& b = comps[j];
			double xi = mix[mixpos++], eta = mix[mixpos++];
			for (int dir = 0; dir < 2; dir++) {
				double ea = dir ? b.eps : a.eps, eb = dir ? a.eps : b.eps;
				double sa = dir ? b.sigma : a.sigma, sb = dir ? a.sigma : b.sigma;
				double epsilon24 = 24. * xi * std::sqrt(ea * eb);
				double sigma2 = eta * .5 * (sa + sb);
				sigma2 *= sigma2;
				double sigperrc2 = sigma2 / (rcLJ * rcLJ);
				double sigperrc6 = sigperrc2 * sigperrc2 * sigperrc2;
				double sh = epsilon24 * (sigperrc6 - sigperrc6 * sigperrc6);
				int k = dir ? j * ncomp + i : i * ncomp + j;
				sp.eps24[k] = epsilon24;
				sp.sig2[k] = sigma2;
				sp.shift6[k] = sh;
			}
		}
	}
	return MDGPU_OK;
}

PairParams pair_params(const Species& sp, double rc, double rc_lj) {
	PairParams hp{};
	hp.ns = sp.n;
	hp.rc2 = rc * rc;
	hp.rclj2 = rc_lj * rc_lj;
	for (int k = 0; k < kMaxSpecies * kMaxSpecies; k++) {
		hp.eps24[k] = sp.eps24[k];
		hp.sig2[k] = sp.sig2[k];
		hp.shift6[k] = sp.shift6[k];
	}
	return hp;
}

int device_max_optin(int device) {
	static std::mutex mu;
	static int known[kMaxDevices] = {};
	const bool cached = device >= 0 && device < kMaxDevices;
	{
		std::lock_guard<std::mutex> lock(mu);
		if (cached && known[device] > 0) return known[device];
	}
	int v = 0;
	if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess || v <= 0)
		v = 48 * 1024;
	std::lock_guard<std::mutex> lock(mu);
	if (cached) known[device] = v;
	return v;
}

int rebuild_prepare(Context* c) {
	const int64_t n = c->n;
	if (c->rb_cap < n) {
		cudaFree(c->rb_slot);
		c->rb_slot = nullptr;
		c->rb_cap = 0;
		MD_CUDA(cudaMalloc(&c->rb_slot, sizeof(int4) * n));
		c->rb_cap = n;
	}
	if (!c->rebuild) {
		MD_CUDA(cudaMalloc(&c->rebuild, sizeof(int)));
		MD_CUDA(cudaMemsetAsync(c->rebuild, 0xff, sizeof(int), c->stream));
		MD_CUDA(cudaMalloc(&c->builds, sizeof(unsigned long long)));
		MD_CUDA(cudaMemsetAsync(c->builds, 0, sizeof(unsigned long long), c->stream));
		MD_CUDA(cudaMalloc(&c->bar, sizeof(unsigned) * 4));
		MD_CUDA(cudaMemsetAsync(c->bar, 0, sizeof(unsigned) * 4, c->stream));
		c->rb_look_cap = 8192;
		MD_CUDA(cudaMalloc(&c->rb_look, sizeof(unsigned long long) * c->rb_look_cap));
		MD_CUDA(cudaMemsetAsync(c->rb_look, 0, sizeof(unsigned long long) * c->rb_look_cap, c->stream));
		MD_CUDA(cudaMalloc(&c->rb_count, sizeof(int32_t) * c->g.ncells));
		MD_CUDA(cudaMemsetAsync(c->rb_count, 0, sizeof(int32_t) * c->g.ncells, c->stream));
	}
	return MDGPU_OK;
}

int request_build(Context* c) {
	k_set_int<<<1, 1, 0, c->stream>>>(c->rebuild, c->step_id);
	count_launches(c, 1);
	MD_CUDA(cudaGetLastError());
	return MDGPU_OK;
}

}  // namespace mdgpu

using namespace mdgpu;

extern "C" {

int mdgpu_create(mdgpu_ctx** out, const double length[3], double cutoff, double lj_cutoff, double cells_in_cutoff,
                 int ncomp, const mdgpu_component* comps, const double* mix, int precision, int device) {
	if (!out || !length || !comps) return MDGPU_ERR_ARG;
	*out = nullptr;
	mdgpu_ctx_full* full = new (std::nothrow) mdgpu_ctx_full();
	if (!full) return MDGPU_ERR_ARG;
	Context* c = &full->pub.c;
	*out = &full->pub;
	if (ncomp < 1 || ncomp > kMaxSpecies) return fail(c, MDGPU_ERR_ARG, "ncomp must be in 1..8");
	if (!(cutoff > 0)) return fail(c, MDGPU_ERR_ARG, "cutoff must be positive");
	if (!(lj_cutoff >= 0)) return fail(c, MDGPU_ERR_ARG, "lj_cutoff must be 0 (= cutoff) or positive");
	if (cells_in_cutoff != 1.0) return fail(c, MDGPU_ERR_ARG, "only cellsInCutoffRadius = 1 is supported");
	if (precision != MDGPU_FP64 && precision != MDGPU_MIXED) return fail(c, MDGPU_ERR_ARG, "unknown precision mode");
	if (ncomp > 1 && !mix) return fail(c, MDGPU_ERR_ARG, "mixing coefficients are required for ncomp > 1");
	int ndev = 0;
	cudaError_t e = cudaGetDeviceCount(&ndev);
	if (e != cudaSuccess || ndev == 0) return fail(c, MDGPU_ERR_CUDA, "no CUDA device is available");
	if (device < 0 || device >= ndev) return fail(c, MDGPU_ERR_ARG, "device index out of range");
	c->device = device;
	c->precision = precision;
	c->rc = cutoff;
	c->rc_lj = lj_cutoff == 0.0 ? cutoff : lj_cutoff;
	MD_CUDA(cudaSetDevice(device));
	MD_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
	{
		int st = setup_grid(length, cutoff, cells_in_cutoff, c->g, c->err);
		if (st) return st;
		st = setup_species(ncomp, comps, mix, c->rc_lj, c->sp, c->err);
		if (st) return st;
	}
	const int64_t ncells = c->g.ncells;
	for (int i = 0; i < ncomp; i++) {
		c->eps[i] = comps[i].eps;
		c->sigma[i] = comps[i].sigma;
		c->do_shift[i] = comps[i].do_shift;
	}
	for (int k = 0; k < ncomp * (ncomp - 1); k++) c->mix[k] = mix[k];
	MD_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
	MD_CUDA(cudaMalloc(&c->cell_count, sizeof(int32_t) * ncells));
	MD_CUDA(cudaMalloc(&c->cell_start, sizeof(int32_t) * (ncells + 1)));
	c->scan_blocks = (ncells + 1023) / 1024;
	MD_CUDA(cudaMalloc(&c->scan_tmp, sizeof(int32_t) * (c->scan_blocks + 1)));
	MD_CUDA(cudaMalloc(&c->scalars, sizeof(double) * 64));
	MD_CUDA(cudaMemset(c->scalars, 0, sizeof(double) * 64));
	MD_CUDA(cudaMalloc(&c->status, sizeof(int)));
	MD_CUDA(cudaMemset(c->status, 0, sizeof(int)));
	MD_CUDA(cudaMalloc(&c->tickets, sizeof(unsigned) * 4));
	MD_CUDA(cudaMemset(c->tickets, 0, sizeof(unsigned) * 4));
	MD_CUDA(cudaMallocHost(&c->h_scalars, sizeof(double) * 64));
	MD_CUDA(cudaMallocHost(&c->h_status, sizeof(int)));
	PairParams hp = pair_params(c->sp, c->rc, c->rc_lj);
	MD_CUDA(cudaMalloc(&c->d_pp, sizeof(PairParams)));
	MD_CUDA(cudaMemcpy(c->d_pp, &hp, sizeof(PairParams), cudaMemcpyHostToDevice));
	c->err.clear();
	return MDGPU_OK;
}

int mdgpu_destroy(mdgpu_ctx* ctx) {
	if (!ctx) return MDGPU_OK;
	mdgpu_ctx_full* full = reinterpret_cast<mdgpu_ctx_full*>(ctx);
	Context* c = &ctx->c;
	cudaSetDevice(c->device);
	if (c->stream) cudaStreamSynchronize(c->stream);
	free_particles(c->p);
	free_particles(c->q);
	cudaFree(c->cell);
	cudaFree(c->rank);
	cudaFree(c->perm);
	cudaFree(c->cell_count);
	cudaFree(c->cell_start);
	cudaFree(c->scan_tmp);
	cudaFree(c->partials);
	cudaFree(c->scalars);
	cudaFree(c->steps_out);
	cudaFree(c->status);
	cudaFree(c->d_pp);
	cudaFree(c->adj);
	free_traj(c);
	cudaFree(c->nbr);
	cudaFree(c->nbr_count);
	cudaFree(c->nbr_in);
	cudaFree(c->nbr_in_count);
	cudaFree(c->prune_st);
	cudaFree(c->r_ref);
	cudaFree(c->rebuild);
	cudaFree(c->builds);
	cudaFree(c->bar);
	cudaFree(c->brick_counts);
	cudaFree(c->brick_list);
	if (c->h_sparse) cudaFreeHost(c->h_sparse);
	cudaFree(c->rb_count);
	cudaFree(c->rb_look);
	cudaFree(c->rb_slot);
	cudaFree(c->tickets);
	cudaFree(c->brick_kind);
	cudaFree(full->x.stage.ptr);
	if (c->h_scalars) cudaFreeHost(c->h_scalars);
	if (c->h_status) cudaFreeHost(c->h_status);
	for (auto& r : full->x.recs) {
		cudaEventDestroy(r.a);
		cudaEventDestroy(r.b);
	}
	for (auto ev : full->x.pool) cudaEventDestroy(ev);
	if (c->stream) cudaStreamDestroy(c->stream);
	delete full;
	return MDGPU_OK;
}

const char* mdgpu_last_error(const mdgpu_ctx* ctx) { return ctx ? ctx->c.err.c_str() : "null context"; }

int mdgpu_set_precision(mdgpu_ctx* ctx, int precision) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (precision != MDGPU_FP64 && precision != MDGPU_MIXED) return fail(c, MDGPU_ERR_ARG, "unknown precision mode");
	c->precision = precision;
	return MDGPU_OK;
}

int mdgpu_set_pair_kernel(mdgpu_ctx* ctx, int kind) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (kind != 0 && kind != 1) return fail(c, MDGPU_ERR_ARG, "pair kernel must be 0 (brick) or 1 (gather)");
	c->pair_kernel = kind;
	return MDGPU_OK;
}

int mdgpu_set_particles(mdgpu_ctx* ctx, int64_t n, const uint64_t* id, const int32_t* cid, const double* r,
                        const double* v, const double* F) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (n <= 0 || n > (int64_t) 0x7fffffff) return fail(c, MDGPU_ERR_ARG, "n must be in 1..2^31-1");
	if (!id || !cid || !r || !v) return fail(c, MDGPU_ERR_ARG, "id, cid, r and v are required");
	Extra* x = extra(c);
	x->species_count.assign(c->sp.n, 0);
	for (int64_t i = 0; i < n; i++) {
		if (cid[i] < 0 || cid[i] >= c->sp.n) return fail(c, MDGPU_ERR_ARG, "component id out of range");
		x->species_count[cid[i]]++;
	}
	// largest cell occupancy (the reference's cell formula after the periodic wrap): sizes the
	// neighbour lists of the Verlet-skin mode
	{
		std::vector<int32_t> occ((size_t) c->g.ncells, 0);
		int mx = 0;
		for (int64_t i = 0; i < n; i++) {
			int64_t cell = 0;
			for (int d = 2; d >= 0; d--) {
				double x = r[3 * i + d];
				if (x < 0.0)
					x += c->g.L[d];
				else if (x >= c->g.L[d])
					x -= c->g.L[d];
				int cc = (int) std::floor((x - c->g.halo_min[d]) / c->g.cell_length[d]) - 1;
				cc = cc < 0 ? 0 : (cc >= c->g.nc[d] ? c->g.nc[d] - 1 : cc);
				cell = cell * c->g.nc[d] + cc;
			}
			mx = std::max(mx, ++occ[(size_t) cell]);
		}
		c->max_occ = mx;
		// the density around a typical molecule: sum occ^2 / sum occ per cell volume
		double s2 = 0.0;
		for (int32_t o : occ) s2 += (double) o * o;
		c->rho_typ = s2 / (double) n / (c->g.cell_length[0] * c->g.cell_length[1] * c->g.cell_length[2]);
	}
	if (c->skin > 0.0) {
		// the skin grid follows the density of the new positions
		Grid gs{};
		std::string err;
		int st = skin_grid(c, c->skin, gs, err);
		if (st) return fail(c, st, "cutoff + skin: " + err);
		c->gs = gs;
	}
	MD_CUDA(cudaSetDevice(c->device));
	MD_CUDA(cudaStreamSynchronize(c->stream));
	if (n > c->cap) {
		free_particles(c->p);
		free_particles(c->q);
		cudaFree(c->cell);
		cudaFree(c->rank);
		cudaFree(c->perm);
		cudaFree(c->partials);
		c->cell = c->rank = c->perm = nullptr;
		c->partials = nullptr;
		MD_CUDA(alloc_particles(c->p, n));
		MD_CUDA(alloc_particles(c->q, n));
		MD_CUDA(cudaMalloc(&c->cell, sizeof(int32_t) * n));
		MD_CUDA(cudaMalloc(&c->rank, sizeof(int32_t) * n));
		MD_CUDA(cudaMalloc(&c->perm, sizeof(int32_t) * n));
		// per-block partials of the widest reduction: per-molecule blocks or one per 2x2x2 brick
		const int64_t bricks = (int64_t) ((c->g.nc[0] + 1) / 2) * ((c->g.nc[1] + 1) / 2) * ((c->g.nc[2] + 1) / 2);
		const int64_t blocks = (n + kReduceBlock - 1) / kReduceBlock;
		c->partial_cap = (blocks > bricks ? blocks : bricks) + 1024;
		MD_CUDA(cudaMalloc(&c->partials, sizeof(double) * 4 * c->partial_cap));
		c->cap = n;
	}
	c->n = n;
	void* st;
	MD_CUDA(staging(c, x->stage, sizeof(double) * 3 * n, &st));
	double* aos = (double*) st;
	MD_CUDA(cudaMemcpyAsync(aos, r, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
	k_load_aos<<<blocks_for(n), kThreads, 0, c->stream>>>(n, aos, nullptr, c->p.rx, c->p.ry, c->p.rz);
	MD_CUDA(cudaMemcpyAsync(aos, v, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
	k_load_aos<<<blocks_for(n), kThreads, 0, c->stream>>>(n, aos, nullptr, c->p.vx, c->p.vy, c->p.vz);
	if (F) {
		MD_CUDA(cudaMemcpyAsync(aos, F, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
		k_load_aos<<<blocks_for(n), kThreads, 0, c->stream>>>(n, aos, nullptr, c->p.fx, c->p.fy, c->p.fz);
	} else {
		MD_CUDA(cudaMemsetAsync(c->p.fx, 0, sizeof(double) * n, c->stream));
		MD_CUDA(cudaMemsetAsync(c->p.fy, 0, sizeof(double) * n, c->stream));
		MD_CUDA(cudaMemsetAsync(c->p.fz, 0, sizeof(double) * n, c->stream));
	}
	MD_CUDA(cudaMemcpyAsync(c->p.id, id, sizeof(uint64_t) * n, cudaMemcpyHostToDevice, c->stream));
	MD_CUDA(cudaMemcpyAsync(c->p.cid, cid, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream));
	k_iota<<<blocks_for(n), kThreads, 0, c->stream>>>(n, c->p.uidx);
	MD_CUDA(cudaGetLastError());
	MD_CUDA(cudaStreamSynchronize(c->stream));
	c->cells_valid = false;
	c->lists_valid = false;
	return MDGPU_OK;
}

int mdgpu_set_state(mdgpu_ctx* ctx, int64_t n, const double* r, const double* v) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (n != c->n) return fail(c, MDGPU_ERR_ARG, "n does not match the loaded molecules");
	MD_CUDA(cudaSetDevice(c->device));
	void* st;
	MD_CUDA(staging(c, extra(c)->stage, sizeof(double) * 6 * n, &st));
	double* aos = (double*) st;
	if (r) {
		MD_CUDA(cudaMemcpyAsync(aos, r, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
		k_load_aos<<<blocks_for(n), kThreads, 0, c->stream>>>(n, aos, c->p.uidx, c->p.rx, c->p.ry, c->p.rz);
		c->cells_valid = false;
	}
	if (v) {
		MD_CUDA(cudaMemcpyAsync(aos + 3 * n, v, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
		k_load_aos<<<blocks_for(n), kThreads, 0, c->stream>>>(n, aos + 3 * n, c->p.uidx, c->p.vx, c->p.vy, c->p.vz);
	}
	count_launches(c, (r ? 1 : 0) + (v ? 1 : 0));
	MD_CUDA(cudaGetLastError());
	return MDGPU_OK;
}

int mdgpu_get_particles(mdgpu_ctx* ctx, int64_t n, uint64_t* id, int32_t* cid, double* r, double* v, double* F) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (n != c->n) return fail(c, MDGPU_ERR_ARG, "n does not match the loaded molecules");
	MD_CUDA(cudaSetDevice(c->device));
	void* st;
	MD_CUDA(staging(c, extra(c)->stage, sizeof(double) * 3 * n, &st));
	double* aos = (double*) st;
	struct {
		double* out;
		double *x, *y, *z;
	} sets[3] = {{r, c->p.rx, c->p.ry, c->p.rz}, {v, c->p.vx, c->p.vy, c->p.vz}, {F, c->p.fx, c->p.fy, c->p.fz}};
	for (auto& s : sets) {
		if (!s.out) continue;
		if (s.out == r)   // positions in [0, L) as after LinkedCells::update (the skin mode defers the wrap)
			k_store_pos<<<blocks_for(n), kThreads, 0, c->stream>>>(n, s.x, s.y, s.z, c->p.uidx, c->g, aos);
		else
			k_store_aos<<<blocks_for(n), kThreads, 0, c->stream>>>(n, s.x, s.y, s.z, c->p.uidx, aos);
		MD_CUDA(cudaMemcpyAsync(s.out, aos, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->stream));
		MD_CUDA(cudaStreamSynchronize(c->stream));
	}
	if (id) {
		k_store_scalar<uint64_t><<<blocks_for(n), kThreads, 0, c->stream>>>(n, c->p.id, c->p.uidx, (uint64_t*) aos);
		MD_CUDA(cudaMemcpyAsync(id, aos, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, c->stream));
		MD_CUDA(cudaStreamSynchronize(c->stream));
	}
	if (cid) {
		k_store_scalar<int32_t><<<blocks_for(n), kThreads, 0, c->stream>>>(n, c->p.cid, c->p.uidx, (int32_t*) aos);
		MD_CUDA(cudaMemcpyAsync(cid, aos, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c->stream));
		MD_CUDA(cudaStreamSynchronize(c->stream));
	}
	MD_CUDA(cudaGetLastError());
	return MDGPU_OK;
}

int mdgpu_num_particles(const mdgpu_ctx* ctx, int64_t* n) {
	if (!ctx || !n) return MDGPU_ERR_ARG;
	*n = ctx->c.n;
	return MDGPU_OK;
}

int mdgpu_get_geometry(const mdgpu_ctx* ctx, int32_t box_cells[3], double cell_length[3], double halo_min[3]) {
	if (!ctx) return MDGPU_ERR_ARG;
	for (int d = 0; d < 3; d++) {
		if (box_cells) box_cells[d] = ctx->c.g.nc[d];
		if (cell_length) cell_length[d] = ctx->c.g.cell_length[d];
		if (halo_min) halo_min[d] = ctx->c.g.halo_min[d];
	}
	return MDGPU_OK;
}

int mdgpu_update(mdgpu_ctx* ctx) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (c->n == 0) return fail(c, MDGPU_ERR_STATE, "no molecules loaded");
	MD_CUDA(cudaSetDevice(c->device));
	MD_CUDA(launch_bin(c, true));
	c->lists_valid = false;
	int st = check_status(c);
	c->cells_valid = (st == MDGPU_OK);
	return st;
}

int mdgpu_get_cell_index(mdgpu_ctx* ctx, int64_t n, int64_t* cell) {
	if (!ctx || !cell) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (n != c->n) return fail(c, MDGPU_ERR_ARG, "n does not match the loaded molecules");
	if (!c->cells_valid) return fail(c, MDGPU_ERR_STATE, "cell structure invalid, call mdgpu_update first");
	MD_CUDA(cudaSetDevice(c->device));
	void* st;
	MD_CUDA(staging(c, extra(c)->stage, sizeof(int64_t) * n, &st));
	k_store_refcell<<<blocks_for(n), kThreads, 0, c->stream>>>(n, c->cell, c->p.uidx, c->g, (int64_t*) st);
	MD_CUDA(cudaMemcpyAsync(cell, st, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, c->stream));
	MD_CUDA(cudaStreamSynchronize(c->stream));
	return MDGPU_OK;
}

int mdgpu_traverse_pairs(mdgpu_ctx* ctx, double* upot, double* virial, double* npairs) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (!c->cells_valid)
		return fail(c, MDGPU_ERR_STATE, "cell structure in the container is invalid, call mdgpu_update first");
	MD_CUDA(cudaSetDevice(c->device));
	MD_CUDA(launch_pairs(c));
	MD_CUDA(cudaMemcpyAsync(c->h_scalars, c->scalars, sizeof(double) * 3, cudaMemcpyDeviceToHost, c->stream));
	int st = check_status(c);
	if (st) return st;
	// ParticlePairs2PotForceAdapter::finish: Upot = Upot6LJ/6, Virial (each pair was seen twice)
	if (upot) *upot = c->h_scalars[0] * 0.5 / 6.;
	if (virial) *virial = c->h_scalars[1] * 0.5;
	if (npairs) *npairs = c->h_scalars[2] * 0.5;
	return MDGPU_OK;
}

int mdgpu_leapfrog_pre(mdgpu_ctx* ctx, double dt, double vcorr) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	MD_CUDA(cudaSetDevice(c->device));
	MD_CUDA(launch_leapfrog_pre(c, dt, vcorr));
	c->cells_valid = false;
	if (pruning(c)) c->lists_valid = false;   // a drift the pruned lists did not see
	return MDGPU_OK;
}

int mdgpu_leapfrog_post(mdgpu_ctx* ctx, double dt_half, double* summv2) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	MD_CUDA(cudaSetDevice(c->device));
	MD_CUDA(launch_leapfrog_post(c, dt_half));
	MD_CUDA(cudaMemcpyAsync(c->h_scalars + 3, c->scalars + 3, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
	int st = check_status(c);
	if (st) return st;
	if (summv2) *summv2 = c->h_scalars[3];
	return MDGPU_OK;
}

int mdgpu_scale_velocities(mdgpu_ctx* ctx, double beta) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	MD_CUDA(cudaSetDevice(c->device));
	MD_CUDA(launch_scale(c, beta));
	return MDGPU_OK;
}

int mdgpu_far_field_correction(mdgpu_ctx* ctx, double* upot_corr, double* virial_corr) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	Extra* x = extra(c);
	if (c->n == 0 || (int) x->species_count.size() != c->sp.n) return fail(c, MDGPU_ERR_STATE, "no molecules loaded");
	// Domain::initFarFieldCorr (Domain.cpp:574-677) for LJ centres at the molecule origin: the
	// TICCu/TICCv terms (CutoffCorrections.cpp:10-32) of every unshifted component pair.
	auto ticc_u = [](int n, double rc, double sigma2) {
		return -std::pow(rc, 2 * n + 3) / (std::pow(sigma2, n) * (2 * n + 3));
	};
	auto ticc_v = [&](int n, double rc, double sigma2) { return 2 * n * ticc_u(n, rc, sigma2); };
	int ns = c->sp.n;
	double U = 0., V = 0.;
	for (int i = 0; i < ns; ++i)
		for (int j = 0; j < ns; ++j) {
			int k = i * ns + j;
			if (c->sp.shift6[k] == 0.0) {
				double fac = double(x->species_count[i]) * double(x->species_count[j]) * c->sp.eps24[k];
				U += fac * (ticc_u(-6, c->rc_lj, c->sp.sig2[k]) - ticc_u(-3, c->rc_lj, c->sp.sig2[k]));
				V += fac * (ticc_v(-6, c->rc_lj, c->sp.sig2[k]) - ticc_v(-3, c->rc_lj, c->sp.sig2[k]));
			}
		}
	double rho = c->n / (c->g.L[0] * c->g.L[1] * c->g.L[2]);
	double fac = M_PI * rho / (3. * c->n);
	if (upot_corr) *upot_corr = U * fac + 0.0;
	if (virial_corr) *virial_corr = V * -fac + 3. * 0.0;
	return MDGPU_OK;
}

namespace {
// Verlet-skin buffers sized for the loaded molecules; the first step after a change of the sort
// order builds the lists.
int skin_prepare(Context* c) {
	const int64_t n = c->n;
	const double rl = c->rc + c->skin;
	const double cell_vol = c->g.cell_length[0] * c->g.cell_length[1] * c->g.cell_length[2];
	const double rho_max = (c->max_occ > 0 ? c->max_occ : 1) / cell_vol;
	int cap = (int) std::ceil(1.25 * 4.18879020478639 * rl * rl * rl * rho_max) + 32;
	cap = (cap + 31) & ~31;
	cap = std::min(cap, 65504);
	if (c->list_n != n || c->list_cap < cap || (pruning(c) && !c->nbr_in)) {
		cudaFree(c->nbr);
		cudaFree(c->nbr_count);
		cudaFree(c->nbr_in);
		cudaFree(c->nbr_in_count);
		cudaFree(c->r_ref);
		c->nbr = nullptr;
		c->nbr_count = nullptr;
		c->nbr_in = nullptr;
		c->nbr_in_count = nullptr;
		c->r_ref = nullptr;
		if (c->list_n == n) cap = std::max(cap, c->list_cap);
		c->list_n = 0;
		MD_CUDA(cudaMalloc(&c->nbr, sizeof(unsigned short) * (size_t) cap * n));
		MD_CUDA(cudaMalloc(&c->nbr_count, sizeof(unsigned short) * n));
		if (pruning(c)) {
			MD_CUDA(cudaMalloc(&c->nbr_in, sizeof(unsigned short) * (size_t) cap * n));
			MD_CUDA(cudaMalloc(&c->nbr_in_count, sizeof(unsigned short) * n));
		}
		MD_CUDA(cudaMalloc(&c->r_ref, sizeof(double) * 3 * n));
		c->list_n = n;
		c->list_cap = cap;
		c->lists_valid = false;
	}
	if (pruning(c) && !c->prune_st) {
		MD_CUDA(cudaMalloc(&c->prune_st, sizeof(PruneState)));
		MD_CUDA(cudaMemsetAsync(c->prune_st, 0, sizeof(PruneState), c->stream));
	}
	{
		const int st = rebuild_prepare(c);
		if (st) return st;
	}
	const int64_t parts = skin_partials_needed(c);
	if (c->brick_kind == nullptr || c->list_n != n || c->lists_valid == false) {
		cudaFree(c->brick_kind);
		cudaFree(c->brick_list);
		c->brick_kind = nullptr;
		c->brick_list = nullptr;
		MD_CUDA(cudaMalloc(&c->brick_kind, parts));
		MD_CUDA(cudaMemsetAsync(c->brick_kind, 0, parts, c->stream));
		MD_CUDA(cudaMalloc(&c->brick_list, sizeof(int32_t) * 2 * parts));
	}
	if (c->partial_cap < parts) {
		MD_CUDA(cudaStreamSynchronize(c->stream));
		cudaFree(c->partials);
		c->partials = nullptr;
		MD_CUDA(cudaMalloc(&c->partials, sizeof(double) * 4 * (parts + 1024)));
		c->partial_cap = parts + 1024;
	}
	if (!c->brick_counts) {
		MD_CUDA(cudaMalloc(&c->brick_counts, sizeof(unsigned) * 4));
		MD_CUDA(cudaMemsetAsync(c->brick_counts, 0, sizeof(unsigned) * 4, c->stream));
		MD_CUDA(cudaMallocHost(&c->h_sparse, sizeof(int)));
		*c->h_sparse = 1;   // unknown until a build has run: launch the sparse-brick kernel
	}
	return MDGPU_OK;
}

// Opens skin-mode step `c->step_id`: asks for a build when the lists do not fit the sort order.
int skin_open_step(Context* c) {
	c->step_id++;
	if (!c->lists_valid) {
		k_set_int<<<1, 1, 0, c->stream>>>(c->rebuild, c->step_id);
		count_launches(c, 1);
		MD_CUDA(cudaGetLastError());
		c->lists_valid = true;
	}
	return MDGPU_OK;
}

// One Simulation::simulateStep hot path, its record written to dst (device).
int enqueue_one(Context* c, double dt, double vcorr, double* dst) {
	if (c->skin > 0.0) {
		int st = skin_prepare(c);
		if (!st) st = skin_open_step(c);
		if (st) return st;
		MD_CUDA(launch_leapfrog_pre(c, dt, vcorr, true));
		MD_CUDA(launch_rebuild(c, c->gs));
		// the closing kick and the record come from the pair kernels
		MD_CUDA(launch_pairs_skin(c, 2, dt, dst));
		return MDGPU_OK;
	} else {
		MD_CUDA(launch_leapfrog_pre(c, dt, vcorr));
		MD_CUDA(launch_bin(c, false));
		c->lists_valid = false;
		MD_CUDA(launch_pairs(c));
		MD_CUDA(launch_leapfrog_post(c, 0.5 * dt));
	}
	MD_CUDA(launch_step_record(c, dst));
	return MDGPU_OK;
}
}  // namespace

int mdgpu_set_skin(mdgpu_ctx* ctx, double skin) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (!(skin >= 0.0) || !(skin < c->rc)) return fail(c, MDGPU_ERR_ARG, "skin must be in [0, cutoff)");
	if (skin > 0.0) {
		Grid gs{};
		std::string err;
		int st = skin_grid(c, skin, gs, err);
		if (st) return fail(c, st, "cutoff + skin: " + err);
		c->gs = gs;
	}
	c->skin = skin;
	c->lists_valid = false;
	return MDGPU_OK;
}

int mdgpu_set_list_prune(mdgpu_ctx* ctx, double prune) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (!(prune >= 0.0) || !(prune < c->rc)) return fail(c, MDGPU_ERR_ARG, "prune must be in [0, cutoff)");
	c->prune = prune;
	c->lists_valid = false;
	return MDGPU_OK;
}

int mdgpu_list_prunes(mdgpu_ctx* ctx, int64_t* prunes) {
	if (!ctx || !prunes) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	*prunes = 0;
	if (!c->prune_st) return MDGPU_OK;
	PruneState st{};
	MD_CUDA(cudaSetDevice(c->device));
	MD_CUDA(cudaMemcpyAsync(&st, c->prune_st, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
	MD_CUDA(cudaStreamSynchronize(c->stream));
	*prunes = (int64_t) st.count;
	return MDGPU_OK;
}

int mdgpu_skin_builds(mdgpu_ctx* ctx, int64_t* builds) {
	if (!ctx || !builds) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	*builds = 0;
	if (!c->builds) return MDGPU_OK;
	unsigned long long v = 0;
	MD_CUDA(cudaSetDevice(c->device));
	MD_CUDA(cudaMemcpyAsync(&v, c->builds, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
	MD_CUDA(cudaStreamSynchronize(c->stream));
	*builds = (int64_t) v;
	return MDGPU_OK;
}

int mdgpu_step(mdgpu_ctx* ctx, double dt, double vcorr, double* out4) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (c->n == 0) return fail(c, MDGPU_ERR_STATE, "no molecules loaded");
	MD_CUDA(cudaSetDevice(c->device));
	int st = enqueue_one(c, dt, vcorr, c->scalars + 8);
	if (st) return st;
	MD_CUDA(cudaMemcpyAsync(c->h_scalars + 8, c->scalars + 8, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->stream));
	st = check_status(c);
	c->cells_valid = (st == MDGPU_OK) && c->skin == 0.0;
	if (st) return st;
	if (out4)
		for (int k = 0; k < 4; k++) out4[k] = c->h_scalars[8 + k];
	return MDGPU_OK;
}

namespace {
int enqueue_steps(Context* c, int32_t nsteps, double dt) {
	if (c->n == 0) return fail(c, MDGPU_ERR_STATE, "no molecules loaded");
	if (nsteps < 0) return fail(c, MDGPU_ERR_ARG, "nsteps must be >= 0");
	MD_CUDA(cudaSetDevice(c->device));
	int64_t need = c->steps_written + nsteps;
	if (need > c->steps_cap) {
		int64_t cap = need > 4096 ? need : 4096;
		double* buf = nullptr;
		MD_CUDA(cudaMalloc(&buf, sizeof(double) * 4 * cap));
		if (c->steps_written > 0)
			MD_CUDA(cudaMemcpyAsync(buf, c->steps_out, sizeof(double) * 4 * c->steps_written, cudaMemcpyDeviceToDevice,
			                        c->stream));
		MD_CUDA(cudaStreamSynchronize(c->stream));
		cudaFree(c->steps_out);
		c->steps_out = buf;
		c->steps_cap = cap;
	}
	if (nsteps == 0) return MDGPU_OK;
	const bool skin = c->skin > 0.0;
	if (skin) {
		// the pair kernels apply the closing kick of step k and the opening kick and drift of step
		// k+1 to the molecules whose forces they sum (new positions into the other buffer, whose
		// role then swaps), and write each step's record
		int st = skin_prepare(c);
		if (st) return st;
		for (int k = 0; k < nsteps; k++) {
			st = skin_open_step(c);
			if (st) return st;
			if (k == 0) MD_CUDA(launch_leapfrog_pre(c, dt, 1.0, true));
			MD_CUDA(launch_rebuild(c, c->gs));
			const bool last = k + 1 == nsteps;
			MD_CUDA(launch_pairs_skin(c, last ? 2 : 1, dt, c->steps_out + 4 * c->steps_written));
			c->steps_written++;
			if (!last) {
				std::swap(c->p.rx, c->q.rx);
				std::swap(c->p.ry, c->q.ry);
				std::swap(c->p.rz, c->q.rz);
			}
		}
		// whether the last build found sparse bricks: decides, for later runs, whether the sparse-brick
		// kernel is launched (the dense kernel evaluates every brick when it is not)
		MD_CUDA(cudaMemcpyAsync(c->h_sparse, c->brick_counts, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
		return MDGPU_OK;
	}
	// the closing kick of step k and the opening kick of step k+1 run as one pass; the record of
	// step k is written after it (its sum m v^2 comes from that pass)
	for (int k = 0; k < nsteps; k++) {
		if (k == 0) {
			MD_CUDA(launch_leapfrog_pre(c, dt, 1.0, false));
		} else {
			MD_CUDA(launch_leapfrog_post_pre(c, dt, false, c->steps_out + 4 * c->steps_written));
			c->steps_written++;
		}
		MD_CUDA(launch_bin(c, false));
		c->lists_valid = false;
		MD_CUDA(launch_pairs(c));
	}
	MD_CUDA(launch_leapfrog_post(c, 0.5 * dt, c->steps_out + 4 * c->steps_written));
	c->steps_written++;
	return MDGPU_OK;
}
}  // namespace

int mdgpu_run(mdgpu_ctx* ctx, int32_t nsteps, double dt, double* per_step) {
	if (!ctx) return MDGPU_ERR_ARG;
	ctx->c.steps_written = 0;  // stream order keeps earlier pending records ahead of these
	int st = mdgpu_run_async(ctx, nsteps, dt);
	if (st) return st;
	return mdgpu_read_steps(ctx, nsteps, per_step);
}

int mdgpu_run_async(mdgpu_ctx* ctx, int32_t nsteps, double dt) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	int st = enqueue_steps(c, nsteps, dt);
	c->cells_valid = (st == MDGPU_OK) && c->skin == 0.0;
	return st;
}

int mdgpu_read_steps(mdgpu_ctx* ctx, int32_t nsteps, double* per_step) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (nsteps < 0 || nsteps > c->steps_written) return fail(c, MDGPU_ERR_ARG, "nsteps exceeds the recorded steps");
	MD_CUDA(cudaSetDevice(c->device));
	if (per_step && nsteps > 0)
		MD_CUDA(cudaMemcpyAsync(per_step, c->steps_out, sizeof(double) * 4 * nsteps, cudaMemcpyDeviceToHost, c->stream));
	int st = check_status(c);
	c->steps_written = 0;
	if (st) c->cells_valid = false;
	return st;
}

int mdgpu_adjoint(mdgpu_ctx* ctx, const double* gF, double gU, double* dL_dr, double* dL_deps, double* dL_dsigma) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (!gF || !dL_dr) return fail(c, MDGPU_ERR_ARG, "gF and dL_dr are required");
	if (!c->cells_valid) return fail(c, MDGPU_ERR_STATE, "cell structure invalid, call mdgpu_update first");
	MD_CUDA(cudaSetDevice(c->device));
	constexpr int KK = kMaxSpecies * kMaxSpecies;
	const int64_t n = c->n;
	const int64_t nb = adjoint_blocks(n);
	const int64_t need = 6 * n + nb * 2 * KK + 2 * KK;
	if (need > c->adj_cap) {
		cudaFree(c->adj);
		c->adj = nullptr;
		MD_CUDA(cudaMalloc(&c->adj, sizeof(double) * need));
		c->adj_cap = need;
	}
	double *gx = c->adj, *gy = gx + n, *gz = gy + n, *ox = gz + n, *oy = ox + n, *oz = oy + n;
	double* pgrad = oz + n;
	double* pout = pgrad + nb * 2 * KK;
	void* st;
	MD_CUDA(staging(c, extra(c)->stage, sizeof(double) * 3 * n, &st));
	double* aos = (double*) st;
	MD_CUDA(cudaMemcpyAsync(aos, gF, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
	k_load_aos<<<blocks_for(n), kThreads, 0, c->stream>>>(n, aos, c->p.uidx, gx, gy, gz);
	count_launches(c, 1);
	MD_CUDA(launch_adjoint(c, gx, gy, gz, gU, ox, oy, oz, pgrad, pout));
	k_store_aos<<<blocks_for(n), kThreads, 0, c->stream>>>(n, ox, oy, oz, c->p.uidx, aos);
	count_launches(c, 1);
	MD_CUDA(cudaMemcpyAsync(dL_dr, aos, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->stream));
	double par[2 * KK];
	MD_CUDA(cudaMemcpyAsync(par, pout, sizeof(par), cudaMemcpyDeviceToHost, c->stream));
	int sts = check_status(c);
	if (sts) return sts;
	// one parameter per unordered component pair: both orientations of the table contribute
	const int ns = c->sp.n;
	for (int a = 0; a < ns; a++)
		for (int b = 0; b < ns; b++) {
			const int ab = a * ns + b, ba = b * ns + a;
			const double ge = a == b ? par[ab] : par[ab] + par[ba];
			const double gs = a == b ? par[KK + ab] : par[KK + ab] + par[KK + ba];
			if (dL_deps) dL_deps[ab] = 24.0 * ge;                            // eps24 = 24 eps_ab
			if (dL_dsigma) dL_dsigma[ab] = 2.0 * std::sqrt(c->sp.sig2[ab]) * gs;  // sig2 = sigma_ab^2
		}
	return MDGPU_OK;
}

int mdgpu_profile_enable(mdgpu_ctx* ctx, int enable) {
	if (!ctx) return MDGPU_ERR_ARG;
	ctx->c.profiling = enable != 0;
	return MDGPU_OK;
}

int mdgpu_profile_read(mdgpu_ctx* ctx, double times_ms[3], int64_t counts[4], int reset) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	Extra* x = extra(c);
	MD_CUDA(cudaSetDevice(c->device));
	MD_CUDA(cudaStreamSynchronize(c->stream));
	for (auto& r : x->recs) {
		float ms = 0;
		MD_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
		c->prof_ms[r.group] += ms;
		x->pool.push_back(r.a);
		x->pool.push_back(r.b);
	}
	x->recs.clear();
	for (int k = 0; k < 3; k++)
		if (times_ms) times_ms[k] = c->prof_ms[k];
	for (int k = 0; k < 4; k++)
		if (counts) counts[k] = c->prof_count[k];
	if (reset) {
		for (int k = 0; k < 3; k++) c->prof_ms[k] = 0;
		for (int k = 0; k < 4; k++) c->prof_count[k] = 0;
	}
	return MDGPU_OK;
}

int mdgpu_get_stream(const mdgpu_ctx* ctx, void** stream) {
	if (!ctx || !stream) return MDGPU_ERR_ARG;
	*stream = (void*) ctx->c.stream;
	return MDGPU_OK;
}

int mdgpu_synchronize(mdgpu_ctx* ctx) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	MD_CUDA(cudaSetDevice(c->device));
	return check_status(c);
}

}  // extern "C"
