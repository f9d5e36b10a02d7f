// Batched ensemble: many independent periodic boxes advanced by ONE persistent kernel per step.
//
// Layout: all boxes' molecules in one structure of arrays, box-major (box b owns the slots
// [poff_b, poff_b + n_b) for the whole run), each box sorted by (cell, id) as the single-box path;
// all boxes' cells in one cell-start array (box b's cells at [coff_b, coff_b + ncells_b)), and all
// boxes' 2x2x2 bricks numbered globally (box b's at [brick0_b, brick0_b + nbricks_b)).
//
// One step = one cooperative launch of k_batch_step, CTAs co-resident, three phases:
//   A  per box (one CTA per box, boxes dealt largest first in a snake order): Leapfrog pre-kick
//      and drift (Molecule::upd_preF, molecules/Molecule.cpp:128-135), periodic wrap and cell
//      index (LinkedCells::update, particleContainer/LinkedCells.cpp:165-180, 535-551; paths
//      relative to madpac/mardyn/), then a counting sort of the box in shared memory: cell counts by
//      shared atomics, block scan, arrival scatter of (id, old slot), per-cell insertion sort by id,
//      gather into the other buffer. The result is the same (cell, id) order as the single-box path.
//   -- grid barrier --
//   B  all bricks of all boxes (static stride or an atomic queue): brick::pairs, the single-box
//      pair kernel's per-brick work, so forces match the single-box path bit for bit.
//   -- grid barrier --
//   C  per box: Leapfrog post-kick (Molecule::upd_postF, Molecule.cpp:193-205), sum m v^2, and the
//      box's brick partials in a fixed order -> the step record {Upot, virial, sum m v^2, pairs}.
// Boxes are independent, so nothing crosses between CTAs except at the two barriers. Each barrier
// wait is bounded by a time limit; a wait that runs out sets the timeout status, the CTA skips the
// rest of the step, and every later launch returns at once until the host has read the status.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "brick.cuh"
#include "grid_sync.cuh"
#include "md_internal.h"
#include "reduce.cuh"

namespace mdgpu {
namespace {

constexpr int kThreads = brick::kThreads;

// Per-box entry of the device table.
struct BatchBox {
	brick::Box bx;
	int64_t poff;
	int32_t n;
	int32_t brick0;
};

struct Kick {
	double pre[kMaxSpecies];    // (0.5 dt) / m
	double post[kMaxSpecies];   // (0.5 dt) / m
	double mass[kMaxSpecies];
};

struct StepArgs {
	brick::Const pc;
	const BatchBox* boxes;
	const int32_t* brick0;      // nboxes + 1
	const int32_t* order;       // boxes by decreasing molecule count
	int nboxes, total_bricks;
	Particles src, dst;
	const PairParams* pp;
	Kick kick;
	double dt;
	int32_t* cstart;
	double* partials;
	double* record;             // nboxes x 4
	int* status;
	unsigned* bar;              // [0] arrivals, [1] generation, [2] brick queue
	int64_t timeout_ns;
	int integrate;              // 0: wrap, bin and forces only (initial force evaluation)
	int dynamic;                // 0: bricks by static stride, 1: by atomic queue
};

// Shared-memory bytes of phase A for a box of n molecules and m cells.
__host__ __device__ inline size_t bin_bytes(int64_t n, int64_t m) {
	size_t o = 0;
	o += sizeof(int) * (size_t) m;                // counts, then fill cursors
	o += sizeof(int) * (size_t) (m + 1);          // starts
	o = (o + 7) & ~size_t(7);
	o += sizeof(uint64_t) * (size_t) n;           // ids in arrival order
	o += sizeof(uint16_t) * (size_t) n;           // cell of each old slot
	o += sizeof(uint16_t) * (size_t) n;           // old slot in arrival order
	return o;
}

// Phase A for box b: kick-drift, wrap, bin and sort src -> dst.
__device__ void bin_box(const StepArgs& a, const BatchBox& B, unsigned char* smem) {
	const Grid& g = B.bx.g;
	const int m = (int) g.ncells, n = B.n, tid = threadIdx.x;
	const int64_t poff = B.poff;
	int* s_count = reinterpret_cast<int*>(smem);
	int* s_start = s_count + m;
	size_t o = (sizeof(int) * (size_t) (2 * m + 1) + 7) & ~size_t(7);
	uint64_t* s_key = reinterpret_cast<uint64_t*>(smem + o);
	uint16_t* s_cell = reinterpret_cast<uint16_t*>(s_key + n);
	uint16_t* s_from = s_cell + n;
	__shared__ int s_wsum[kThreads / 32];

	for (int c = tid; c < m; c += kThreads) s_count[c] = 0;
	__syncthreads();
	bool bad = false;
	for (int t = tid; t < n; t += kThreads) {
		const int64_t i = poff + t;
		double r[3] = {a.src.rx[i], a.src.ry[i], a.src.rz[i]};
		if (a.integrate) {
			// Molecule::upd_preF with vcorr = 1: v = vcorr*v + dtInv2m*F; r += dt*v
			const double k = a.kick.pre[a.src.cid[i]];
			double* vp[3] = {a.src.vx, a.src.vy, a.src.vz};
			const double* fp[3] = {a.src.fx, a.src.fy, a.src.fz};
			for (int d = 0; d < 3; d++) {
				const double v = __dadd_rn(__dmul_rn(1.0, vp[d][i]), __dmul_rn(k, fp[d][i]));
				vp[d][i] = v;
				r[d] = __dadd_rn(r[d], __dmul_rn(a.dt, v));
			}
		}
		int ci[3];
		for (int d = 0; d < 3; d++) {
			const double x = r[d];
			double xw = x;
			if (x < 0.0)
				xw = __dadd_rn(x, g.L[d]);
			else if (x >= g.L[d])
				xw = __dsub_rn(x, g.L[d]);
			r[d] = xw;
			int c = (int) floor(__ddiv_rn(__dsub_rn(xw, g.halo_min[d]), g.cell_length[d]));
			if (c < 1 || c > g.nc[d]) {
				bad = true;
				c = c < 1 ? 1 : g.nc[d];
			}
			ci[d] = c - 1;
			if (!(x == x)) bad = true;
		}
		a.src.rx[i] = r[0];
		a.src.ry[i] = r[1];
		a.src.rz[i] = r[2];
		const int c = (ci[2] * g.nc[1] + ci[1]) * g.nc[0] + ci[0];
		s_cell[t] = (uint16_t) c;
		atomicAdd(&s_count[c], 1);
	}
	if (bad) atomicOr(a.status, kStatusOutsideHalo);
	__syncthreads();
	// exclusive scan of the cell counts: contiguous chunks per thread, then a block scan of the sums
	{
		const int per = (m + kThreads - 1) / kThreads;
		const int lo = min(tid * per, m), hi = min(lo + per, m);
		int sum = 0;
		for (int k = lo; k < hi; k++) sum += s_count[k];
		const int lane = tid & 31, warp = tid >> 5;
		int inc = sum;
		for (int of = 1; of < 32; of <<= 1) {
			const int y = __shfl_up_sync(0xffffffffu, inc, of);
			if (lane >= of) inc += y;
		}
		if (lane == 31) s_wsum[warp] = inc;
		__syncthreads();
		if (warp == 0) {
			int w = lane < kThreads / 32 ? s_wsum[lane] : 0;
			for (int of = 1; of < kThreads / 32; of <<= 1) {
				const int y = __shfl_up_sync(0xffffffffu, w, of);
				if (lane >= of) w += y;
			}
			if (lane < kThreads / 32) s_wsum[lane] = w;
		}
		__syncthreads();
		int excl = inc - sum + (warp > 0 ? s_wsum[warp - 1] : 0);
		for (int k = lo; k < hi; k++) {
			s_start[k] = excl;
			excl += s_count[k];
		}
		if (tid == kThreads - 1) s_start[m] = excl;
	}
	__syncthreads();
	for (int c = tid; c <= m; c += kThreads) {
		a.cstart[B.bx.coff + c] = (int32_t) (poff + s_start[c]);
		if (c < m) s_count[c] = s_start[c];
	}
	__syncthreads();
	// arrival scatter of (id, old slot)
	for (int t = tid; t < n; t += kThreads) {
		const int pos = atomicAdd(&s_count[s_cell[t]], 1);
		s_key[pos] = a.src.id[poff + t];
		s_from[pos] = (uint16_t) t;
	}
	__syncthreads();
	// per-cell insertion sort by (id, old slot)
	for (int c = tid; c < m; c += kThreads) {
		const int s = s_start[c], e = s_start[c + 1];
		for (int k = s + 1; k < e; k++) {
			const uint64_t key = s_key[k];
			const uint16_t fr = s_from[k];
			int j = k - 1;
			while (j >= s && (s_key[j] > key || (s_key[j] == key && s_from[j] > fr))) {
				s_key[j + 1] = s_key[j];
				s_from[j + 1] = s_from[j];
				j--;
			}
			s_key[j + 1] = key;
			s_from[j + 1] = fr;
		}
	}
	__syncthreads();
	// gather into the new order
	for (int f = tid; f < n; f += kThreads) {
		const int64_t from = poff + s_from[f], to = poff + f;
		a.dst.rx[to] = a.src.rx[from];
		a.dst.ry[to] = a.src.ry[from];
		a.dst.rz[to] = a.src.rz[from];
		a.dst.vx[to] = a.src.vx[from];
		a.dst.vy[to] = a.src.vy[from];
		a.dst.vz[to] = a.src.vz[from];
		a.dst.id[to] = s_key[f];
		a.dst.cid[to] = a.src.cid[from];
		a.dst.uidx[to] = a.src.uidx[from];
	}
	__syncthreads();
}

// Phase C for box b: post-kick, sum m v^2, the box's brick partials -> record.
__device__ void finish_box(const StepArgs& a, const BatchBox& B, int b) {
	__shared__ double s_w[kThreads / 32];
	const int tid = threadIdx.x;
	double mv2 = 0.0;
	bool bad = false;
	for (int t = tid; t < B.n; t += kThreads) {
		const int64_t i = B.poff + t;
		const int ty = a.dst.cid[i];
		double vx = a.dst.vx[i], vy = a.dst.vy[i], vz = a.dst.vz[i];
		if (a.integrate) {
			const double k = a.kick.post[ty];
			vx = __dadd_rn(vx, __dmul_rn(k, a.dst.fx[i]));
			vy = __dadd_rn(vy, __dmul_rn(k, a.dst.fy[i]));
			vz = __dadd_rn(vz, __dmul_rn(k, a.dst.fz[i]));
			a.dst.vx[i] = vx;
			a.dst.vy[i] = vy;
			a.dst.vz[i] = vz;
		}
		const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
		mv2 += __dmul_rn(a.kick.mass[ty], v2);
		if (!(v2 == v2) || isinf(v2)) bad = true;
	}
	if (bad) atomicOr(a.status, kStatusNonFinite);
	mv2 = warp_sum(mv2);
	if ((tid & 31) == 0) s_w[tid >> 5] = mv2;
	__syncthreads();
	if (tid == 0) {
		double s = 0.0;
		for (int w = 0; w < kThreads / 32; w++) s += s_w[w];
		double U = 0.0, W = 0.0, NP = 0.0;
		const int nbr = B.bx.nb[0] * B.bx.nb[1] * B.bx.nb[2];
		for (int k = 0; k < nbr; k++) {
			const double* q = a.partials + 4 * (int64_t) (B.brick0 + k);
			U += q[0];
			W += q[1];
			NP += q[2];
		}
		double* rec = a.record + 4 * (int64_t) b;
		rec[0] = U * 0.5 / 6.;
		rec[1] = W * 0.5;
		rec[2] = s;
		rec[3] = NP * 0.5;
	}
	__syncthreads();
}

// Boxes of this CTA: j-th in the snake order over boxes sorted by decreasing size.
template <typename F>
__device__ __forceinline__ void for_my_boxes(const StepArgs& a, F&& f) {
	const int G = gridDim.x;
	for (int r = 0; r * G < a.nboxes; r++) {
		const int j = (r & 1) ? (r + 1) * G - 1 - (int) blockIdx.x : r * G + (int) blockIdx.x;
		if (j < a.nboxes) f(a.order[j]);
	}
}

template <bool kFP64, bool kSingle, bool kLjIsRc, int kCap>
__global__ void __launch_bounds__(kThreads) k_batch_step(StepArgs a) {
	extern __shared__ __align__(16) unsigned char smem[];
	__shared__ int s_flag;
	__shared__ int s_item;
	if (threadIdx.x == 0) s_flag = (*((volatile int*) a.status) & kStatusTimeout) ? 1 : 0;
	__syncthreads();
	if (s_flag) return;   // an earlier launch gave up at a barrier: do nothing until the host resets

	// ---- A: per box kick-drift, wrap, bin, sort ----------------------------------------------
	for_my_boxes(a, [&](int b) { bin_box(a, a.boxes[b], smem); });
	if (!grid_barrier(a.bar, a.status, a.timeout_ns, &s_flag)) return;

	// ---- B: pair forces of every brick -------------------------------------------------------
	const brick::SmemLayout L = brick::layout(a.pc.s_cap, kFP64, kCap);
	brick::load_params(smem, L, a.pp, a.pc.ns);
	__syncthreads();
	auto do_brick = [&](int item) {
		int lo = 0, hi = a.nboxes - 1;   // box with brick0[box] <= item < brick0[box + 1]
		while (lo < hi) {
			const int mid = (lo + hi + 1) >> 1;
			if (a.brick0[mid] <= item)
				lo = mid;
			else
				hi = mid - 1;
		}
		const BatchBox& B = a.boxes[lo];
		brick::pairs<kFP64, kSingle, kLjIsRc, kCap>(a.pc, B.bx, item - B.brick0, item, smem, a.dst.rx, a.dst.ry,
		                                            a.dst.rz, a.dst.cid, a.cstart, a.dst.fx, a.dst.fy, a.dst.fz,
		                                            a.partials, a.status);
		__syncthreads();
	};
	if (a.dynamic) {
		for (;;) {
			if (threadIdx.x == 0) s_item = (int) atomicAdd(a.bar + 2, 1u);
			__syncthreads();
			const int item = s_item;
			__syncthreads();
			if (item >= a.total_bricks) break;
			do_brick(item);
		}
	} else {
		for (int item = blockIdx.x; item < a.total_bricks; item += gridDim.x) do_brick(item);
	}
	if (!grid_barrier(a.bar, a.status, a.timeout_ns, &s_flag)) return;

	// ---- C: per box post-kick and records ----------------------------------------------------
	if (blockIdx.x == 0 && threadIdx.x == 0) a.bar[2] = 0u;   // queue is idle until the next launch
	for_my_boxes(a, [&](int b) { finish_box(a, a.boxes[b], b); });
}

using StepKernel = void (*)(StepArgs);

template <int kCap>
StepKernel pick(bool fp64, bool single, bool ljrc) {
	if (fp64) return single ? k_batch_step<true, true, false, kCap> : k_batch_step<true, false, false, kCap>;
	if (ljrc) return single ? k_batch_step<false, true, true, kCap> : k_batch_step<false, false, true, kCap>;
	return single ? k_batch_step<false, true, false, kCap> : k_batch_step<false, false, false, kCap>;
}

__global__ void k_load3(int64_t n, const double* __restrict__ aos, double* x, double* y, double* z) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	x[s] = aos[3 * s];
	y[s] = aos[3 * s + 1];
	z[s] = aos[3 * s + 2];
}

__global__ void k_store3(int64_t n, const double* x, const double* y, const double* z, const int32_t* uidx,
                         double* __restrict__ aos) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const int64_t u = uidx[s];
	aos[3 * u] = x[s];
	aos[3 * u + 1] = y[s];
	aos[3 * u + 2] = z[s];
}

template <typename T>
__global__ void k_store1(int64_t n, const T* x, const int32_t* uidx, T* __restrict__ out) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n) out[uidx[s]] = x[s];
}

__global__ void k_iota32(int64_t n, int32_t* a) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n) a[s] = (int32_t) s;
}

inline unsigned blocks(int64_t n) { return (unsigned) ((n + kThreads - 1) / kThreads); }

struct Tiles {
	int cap = 64, ctas = 2, dynamic = 1;
	bool operator==(const Tiles& o) const { return cap == o.cap && ctas == o.ctas && dynamic == o.dynamic; }
};

struct GraphEntry {
	int nsteps, parity;
	double dt;
	Tiles t;
	cudaGraphExec_t exec;
};

}  // namespace

struct Batch {
	int device = 0;
	cudaStream_t stream = nullptr;
	int precision = MDGPU_FP64;
	double rc = 0, rc_lj = 0;
	Species sp{};
	int nboxes = 0;
	int64_t ntotal = 0;
	int total_cells = 0, total_bricks = 0;
	std::vector<BatchBox> h_boxes;
	std::vector<int32_t> h_order;
	std::string err;
	Particles buf[2]{};
	int cur = 0;
	bool loaded = false, prepared = false;
	int32_t* cstart = nullptr;
	double* partials = nullptr;
	double* records = nullptr;
	int64_t records_cap = 0;      // in steps
	double* prep = nullptr;       // nboxes x 4
	int* status = nullptr;
	int* h_status = nullptr;
	unsigned* bar = nullptr;
	PairParams* d_pp = nullptr;
	BatchBox* d_boxes = nullptr;
	int32_t* d_brick0 = nullptr;
	int32_t* d_order = nullptr;
	double* stage = nullptr;
	size_t stage_bytes = 0;
	Particles backup{};
	bool backup_alloc = false;
	size_t max_bin_bytes = 0;
	Tiles tiles;
	int64_t timeout_ns = 2000000000LL;
	std::vector<GraphEntry> graphs;
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;
	double last_ms = 0.0;
	int num_sms = 0, max_optin = 0;
};

namespace {

int bfail(Batch* b, int code, const std::string& msg) {
	b->err = msg;
	return code;
}

#define B_CUDA(call)                                                            \
	do {                                                                        \
		cudaError_t e_ = (call);                                                \
		if (e_ != cudaSuccess) {                                                \
			b->err = std::string(#call) + ": " + cudaGetErrorString(e_);        \
			return MDGPU_ERR_CUDA;                                              \
		}                                                                       \
	} while (0)

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

void free_particles(Particles& p) {
	void* a[] = {p.rx, p.ry, p.rz, p.vx, p.vy, p.vz, p.fx, p.fy, p.fz, p.id, p.cid, p.uidx};
	for (void* x : a) cudaFree(x);
	p = Particles{};
}

cudaError_t copy_particles(Particles& dst, const Particles& src, int64_t n, cudaStream_t s) {
	const size_t d = sizeof(double) * n;
	double* sd[] = {src.rx, src.ry, src.rz, src.vx, src.vy, src.vz, src.fx, src.fy, src.fz};
	double* dd[] = {dst.rx, dst.ry, dst.rz, dst.vx, dst.vy, dst.vz, dst.fx, dst.fy, dst.fz};
	for (int k = 0; k < 9; k++) {
		cudaError_t e = cudaMemcpyAsync(dd[k], sd[k], d, cudaMemcpyDeviceToDevice, s);
		if (e != cudaSuccess) return e;
	}
	cudaError_t e = cudaMemcpyAsync(dst.id, src.id, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s);
	if (e == cudaSuccess) e = cudaMemcpyAsync(dst.cid, src.cid, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s);
	if (e == cudaSuccess) e = cudaMemcpyAsync(dst.uidx, src.uidx, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s);
	return e;
}

int check_status(Batch* b) {
	B_CUDA(cudaMemcpyAsync(b->h_status, b->status, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
	B_CUDA(cudaStreamSynchronize(b->stream));
	const int st = *b->h_status;
	if (st == 0) return MDGPU_OK;
	B_CUDA(cudaMemsetAsync(b->status, 0, sizeof(int), b->stream));
	if (st & kStatusTimeout) {
		// barrier words may be left mid-count: start them again
		B_CUDA(cudaMemsetAsync(b->bar, 0, sizeof(unsigned) * 4, b->stream));
		B_CUDA(cudaStreamSynchronize(b->stream));
		b->prepared = false;
		return bfail(b, MDGPU_ERR_TIMEOUT, "a grid-barrier wait of the batched step kernel ran out");
	}
	b->prepared = false;
	if (st & kStatusOutsideHalo)
		return bfail(b, MDGPU_ERR_OUTSIDE_HALO, "a molecule is outside the halo box (moved more than one cell in a step)");
	if (st & kStatusSamePosition) return bfail(b, MDGPU_ERR_SAME_POSITION, "two molecules have the same position");
	if (st & kStatusNonFinite) return bfail(b, MDGPU_ERR_NONFINITE, "non-finite force or velocity");
	if (st & kStatusCapacity) return bfail(b, MDGPU_ERR_CAPACITY, "a device buffer is too small for the workload");
	return bfail(b, MDGPU_ERR_CUDA, "unknown device status");
}

// Launch geometry of a tile shape: kernel, grid, dynamic shared memory.
struct Launch {
	StepKernel kern;
	int grid;
	size_t smem;
	brick::Const pc;
};

int plan(Batch* b, const Tiles& t, Launch& L) {
	const bool fp64 = b->precision == MDGPU_FP64;
	const bool single = b->sp.n == 1, ljrc = b->rc_lj == b->rc;
	L.kern = t.cap == 32 ? pick<32>(fp64, single, ljrc) : pick<64>(fp64, single, ljrc);
	// per-CTA shared memory: the SM's 228 KB split between the CTAs, 1 KB reserved per CTA, static
	// shared memory of the kernel and a margin
	size_t budget = t.ctas == 1 ? 220 * 1024 : 110 * 1024;
	if (budget > (size_t) b->max_optin) budget = (size_t) b->max_optin;
	if (b->max_bin_bytes > budget) return bfail(b, MDGPU_ERR_CAPACITY, "a box is too large for this tile shape");
	const int s_cap = brick::capacity_for(budget, fp64, t.cap);
	L.pc = brick::make_const(b->sp.n, s_cap, b->rc, b->rc_lj);
	L.smem = std::max(brick::layout(s_cap, fp64, t.cap).total, b->max_bin_bytes);
	B_CUDA(cudaFuncSetAttribute(L.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) L.smem));
	int per_sm = 0;
	B_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, L.kern, kThreads, L.smem));
	if (per_sm < 1) return bfail(b, MDGPU_ERR_CAPACITY, "the batched step kernel does not fit on an SM");
	per_sm = std::min(per_sm, t.ctas);
	L.grid = per_sm * b->num_sms;
	return MDGPU_OK;
}

StepArgs args(Batch* b, const Launch& L, int src, int integrate, double dt, double* record) {
	StepArgs a{};
	a.pc = L.pc;
	a.boxes = b->d_boxes;
	a.brick0 = b->d_brick0;
	a.order = b->d_order;
	a.nboxes = b->nboxes;
	a.total_bricks = b->total_bricks;
	a.src = b->buf[src];
	a.dst = b->buf[1 - src];
	a.pp = b->d_pp;
	for (int k = 0; k < b->sp.n; k++) {
		a.kick.pre[k] = (.5 * dt) / b->sp.mass[k];
		a.kick.post[k] = (0.5 * dt) / b->sp.mass[k];
		a.kick.mass[k] = b->sp.mass[k];
	}
	a.dt = dt;
	a.cstart = b->cstart;
	a.partials = b->partials;
	a.record = record;
	a.status = b->status;
	a.bar = b->bar;
	a.timeout_ns = b->timeout_ns;
	a.integrate = integrate;
	a.dynamic = b->tiles.dynamic;
	return a;
}

cudaError_t launch_step(Batch* b, const Launch& L, const StepArgs& a) {
	cudaLaunchConfig_t cfg{};
	cfg.gridDim = dim3((unsigned) L.grid);
	cfg.blockDim = dim3(kThreads);
	cfg.dynamicSmemBytes = L.smem;
	cfg.stream = b->stream;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeCooperative;
	attr[0].val.cooperative = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	return cudaLaunchKernelEx(&cfg, L.kern, a);
}

int ensure_records(Batch* b, int64_t nsteps) {
	if (nsteps <= b->records_cap) return MDGPU_OK;
	cudaFree(b->records);
	b->records = nullptr;
	b->records_cap = 0;
	for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);   // graphs hold the old record pointers
	b->graphs.clear();
	B_CUDA(cudaMalloc(&b->records, sizeof(double) * 4 * b->nboxes * nsteps));
	b->records_cap = nsteps;
	return MDGPU_OK;
}

// nsteps launches from buffer parity b->cur, captured once per (nsteps, parity, tiles) and replayed.
int run_steps(Batch* b, int32_t nsteps, double dt) {
	Launch L;
	int st = plan(b, b->tiles, L);
	if (st) return st;
	st = ensure_records(b, nsteps);
	if (st) return st;
	GraphEntry* ge = nullptr;
	// dt is baked into the launches' arguments, so it is part of the key
	for (auto& g : b->graphs)
		if (g.nsteps == nsteps && g.parity == b->cur && g.dt == dt && g.t == b->tiles) ge = &g;
	if (!ge) {
		cudaGraph_t graph = nullptr;
		B_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
		cudaError_t e = cudaSuccess;
		int src = b->cur;
		for (int k = 0; k < nsteps && e == cudaSuccess; k++) {
			const StepArgs a = args(b, L, src, 1, dt, b->records + (int64_t) 4 * b->nboxes * k);
			e = launch_step(b, L, a);
			src = 1 - src;
		}
		cudaError_t e2 = cudaStreamEndCapture(b->stream, &graph);
		if (e != cudaSuccess || e2 != cudaSuccess) {
			if (graph) cudaGraphDestroy(graph);
			b->err = std::string("capturing the batched step graph: ") + cudaGetErrorString(e != cudaSuccess ? e : e2);
			return MDGPU_ERR_CUDA;
		}
		cudaGraphExec_t exec = nullptr;
		e = cudaGraphInstantiate(&exec, graph, 0);
		cudaGraphDestroy(graph);
		if (e != cudaSuccess) {
			b->err = std::string("instantiating the batched step graph: ") + cudaGetErrorString(e);
			return MDGPU_ERR_CUDA;
		}
		b->graphs.push_back({nsteps, b->cur, dt, b->tiles, exec});
		ge = &b->graphs.back();
	}
	B_CUDA(cudaEventRecord(b->ev0, b->stream));
	B_CUDA(cudaGraphLaunch(ge->exec, b->stream));
	B_CUDA(cudaEventRecord(b->ev1, b->stream));
	if (nsteps & 1) b->cur = 1 - b->cur;
	return MDGPU_OK;
}

}  // namespace
}  // namespace mdgpu

struct mdgpu_batch {
	mdgpu::Batch b;
};

using namespace mdgpu;

extern "C" {

int mdgpu_batch_create(mdgpu_batch** out, int32_t nboxes, const double* lengths, const int64_t* counts, double cutoff,
                       double lj_cutoff, double cells_in_cutoff, int ncomp, const mdgpu_component* comps,
                       const double* mix, int precision, int device) {
	if (!out || !lengths || !counts || !comps) return MDGPU_ERR_ARG;
	*out = nullptr;
	mdgpu_batch* h = new (std::nothrow) mdgpu_batch();
	if (!h) return MDGPU_ERR_ARG;
	*out = h;
	Batch* b = &h->b;
	if (nboxes < 1) return bfail(b, MDGPU_ERR_ARG, "nboxes must be >= 1");
	if (ncomp < 1 || ncomp > kMaxSpecies) return bfail(b, MDGPU_ERR_ARG, "ncomp must be in 1..8");
	if (!(cutoff > 0)) return bfail(b, MDGPU_ERR_ARG, "cutoff must be positive");
	if (cells_in_cutoff != 1.0) return bfail(b, MDGPU_ERR_ARG, "only cellsInCutoffRadius = 1 is supported");
	if (precision != MDGPU_FP64 && precision != MDGPU_MIXED) return bfail(b, MDGPU_ERR_ARG, "unknown precision mode");
	if (ncomp > 1 && !mix) return bfail(b, MDGPU_ERR_ARG, "mixing coefficients are required for ncomp > 1");
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return bfail(b, MDGPU_ERR_CUDA, "no CUDA device is available");
	if (device < 0 || device >= ndev) return bfail(b, MDGPU_ERR_ARG, "device index out of range");
	b->device = device;
	b->precision = precision;
	b->rc = cutoff;
	b->rc_lj = lj_cutoff == 0.0 ? cutoff : lj_cutoff;
	b->nboxes = nboxes;
	int st = setup_species(ncomp, comps, mix, b->rc_lj, b->sp, b->err);
	if (st) return st;
	b->h_boxes.resize(nboxes);
	int64_t poff = 0, coff = 0, brick0 = 0;
	std::vector<int32_t> h_brick0(nboxes + 1);
	for (int k = 0; k < nboxes; k++) {
		if (counts[k] < 1) return bfail(b, MDGPU_ERR_ARG, "every box needs at least one molecule");
		Grid g{};
		st = setup_grid(lengths + 3 * k, cutoff, cells_in_cutoff, g, b->err);
		if (st) {
			b->err = "box " + std::to_string(k) + ": " + b->err;
			return st;
		}
		if (g.ncells > 65535) return bfail(b, MDGPU_ERR_CAPACITY, "box " + std::to_string(k) + " has more than 65535 cells");
		if (counts[k] > 65535) return bfail(b, MDGPU_ERR_CAPACITY, "box " + std::to_string(k) + " has more than 65535 molecules");
		BatchBox& B = b->h_boxes[k];
		brick::init_box(B.bx, g, cutoff, (int32_t) coff);
		B.poff = poff;
		B.n = (int32_t) counts[k];
		B.brick0 = (int32_t) brick0;
		h_brick0[k] = (int32_t) brick0;
		b->max_bin_bytes = std::max(b->max_bin_bytes, bin_bytes(counts[k], g.ncells));
		poff += counts[k];
		coff += g.ncells;
		brick0 += (int64_t) B.bx.nb[0] * B.bx.nb[1] * B.bx.nb[2];
		if (poff >= (1LL << 28) || coff >= (1LL << 30) || brick0 >= (1LL << 30))
			return bfail(b, MDGPU_ERR_CAPACITY, "the batch exceeds 2^28 molecules or 2^30 cells/bricks");
	}
	h_brick0[nboxes] = (int32_t) brick0;
	b->ntotal = poff;
	b->total_cells = (int) coff;
	b->total_bricks = (int) brick0;
	b->h_order.resize(nboxes);
	for (int k = 0; k < nboxes; k++) b->h_order[k] = k;
	std::stable_sort(b->h_order.begin(), b->h_order.end(),
	                 [&](int x, int y) { return b->h_boxes[x].n > b->h_boxes[y].n; });

	B_CUDA(cudaSetDevice(device));
	B_CUDA(cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device));
	B_CUDA(cudaDeviceGetAttribute(&b->max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
	if (b->max_bin_bytes > (size_t) b->max_optin - 8192)
		return bfail(b, MDGPU_ERR_CAPACITY, "a box's cell sort does not fit in shared memory");
	if (b->max_bin_bytes > 110 * 1024) b->tiles.ctas = 1;
	int coop = 0;
	B_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
	if (!coop) return bfail(b, MDGPU_ERR_CUDA, "the device does not support cooperative launches");
	B_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
	B_CUDA(cudaEventCreate(&b->ev0));
	B_CUDA(cudaEventCreate(&b->ev1));
	for (int k = 0; k < 2; k++) B_CUDA(alloc_particles(b->buf[k], b->ntotal));
	B_CUDA(cudaMalloc(&b->cstart, sizeof(int32_t) * (b->total_cells + 1)));
	B_CUDA(cudaMalloc(&b->partials, sizeof(double) * 4 * b->total_bricks));
	B_CUDA(cudaMalloc(&b->prep, sizeof(double) * 4 * nboxes));
	B_CUDA(cudaMalloc(&b->status, sizeof(int)));
	B_CUDA(cudaMemset(b->status, 0, sizeof(int)));
	B_CUDA(cudaMallocHost(&b->h_status, sizeof(int)));
	B_CUDA(cudaMalloc(&b->bar, sizeof(unsigned) * 4));
	B_CUDA(cudaMemset(b->bar, 0, sizeof(unsigned) * 4));
	PairParams hp = pair_params(b->sp, b->rc, b->rc_lj);
	B_CUDA(cudaMalloc(&b->d_pp, sizeof(PairParams)));
	B_CUDA(cudaMemcpy(b->d_pp, &hp, sizeof(PairParams), cudaMemcpyHostToDevice));
	B_CUDA(cudaMalloc(&b->d_boxes, sizeof(BatchBox) * nboxes));
	B_CUDA(cudaMemcpy(b->d_boxes, b->h_boxes.data(), sizeof(BatchBox) * nboxes, cudaMemcpyHostToDevice));
	B_CUDA(cudaMalloc(&b->d_brick0, sizeof(int32_t) * (nboxes + 1)));
	B_CUDA(cudaMemcpy(b->d_brick0, h_brick0.data(), sizeof(int32_t) * (nboxes + 1), cudaMemcpyHostToDevice));
	B_CUDA(cudaMalloc(&b->d_order, sizeof(int32_t) * nboxes));
	B_CUDA(cudaMemcpy(b->d_order, b->h_order.data(), sizeof(int32_t) * nboxes, cudaMemcpyHostToDevice));
	b->err.clear();
	return MDGPU_OK;
}

int mdgpu_batch_destroy(mdgpu_batch* h) {
	if (!h) return MDGPU_OK;
	Batch* b = &h->b;
	cudaSetDevice(b->device);
	if (b->stream) cudaStreamSynchronize(b->stream);
	for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);
	for (int k = 0; k < 2; k++) free_particles(b->buf[k]);
	if (b->backup_alloc) free_particles(b->backup);
	void* bufs[] = {b->cstart, b->partials, b->records, b->prep, b->status, b->bar, b->d_pp, b->d_boxes,
	                b->d_brick0, b->d_order, b->stage};
	for (void* x : bufs) cudaFree(x);
	if (b->h_status) cudaFreeHost(b->h_status);
	if (b->ev0) cudaEventDestroy(b->ev0);
	if (b->ev1) cudaEventDestroy(b->ev1);
	if (b->stream) cudaStreamDestroy(b->stream);
	delete h;
	return MDGPU_OK;
}

const char* mdgpu_batch_last_error(const mdgpu_batch* h) { return h ? h->b.err.c_str() : "null batch"; }

int mdgpu_batch_set_particles(mdgpu_batch* h, int64_t ntotal, const uint64_t* id, const int32_t* cid, const double* r,
                              const double* v) {
	if (!h) return MDGPU_ERR_ARG;
	Batch* b = &h->b;
	if (ntotal != b->ntotal) return bfail(b, MDGPU_ERR_ARG, "ntotal must equal the sum of the box counts");
	if (!id || !cid || !r || !v) return bfail(b, MDGPU_ERR_ARG, "id, cid, r and v are required");
	for (int64_t i = 0; i < ntotal; i++)
		if (cid[i] < 0 || cid[i] >= b->sp.n) return bfail(b, MDGPU_ERR_ARG, "component id out of range");
	B_CUDA(cudaSetDevice(b->device));
	const size_t need = sizeof(double) * 3 * ntotal;
	if (b->stage_bytes < need) {
		cudaFree(b->stage);
		b->stage = nullptr;
		b->stage_bytes = 0;
		B_CUDA(cudaMalloc(&b->stage, need));
		b->stage_bytes = need;
	}
	b->cur = 0;
	Particles& p = b->buf[0];
	B_CUDA(cudaMemcpyAsync(b->stage, r, need, cudaMemcpyHostToDevice, b->stream));
	k_load3<<<blocks(ntotal), kThreads, 0, b->stream>>>(ntotal, b->stage, p.rx, p.ry, p.rz);
	B_CUDA(cudaMemcpyAsync(b->stage, v, need, cudaMemcpyHostToDevice, b->stream));
	k_load3<<<blocks(ntotal), kThreads, 0, b->stream>>>(ntotal, b->stage, p.vx, p.vy, p.vz);
	B_CUDA(cudaMemsetAsync(p.fx, 0, sizeof(double) * ntotal, b->stream));
	B_CUDA(cudaMemsetAsync(p.fy, 0, sizeof(double) * ntotal, b->stream));
	B_CUDA(cudaMemsetAsync(p.fz, 0, sizeof(double) * ntotal, b->stream));
	B_CUDA(cudaMemcpyAsync(p.id, id, sizeof(uint64_t) * ntotal, cudaMemcpyHostToDevice, b->stream));
	B_CUDA(cudaMemcpyAsync(p.cid, cid, sizeof(int32_t) * ntotal, cudaMemcpyHostToDevice, b->stream));
	k_iota32<<<blocks(ntotal), kThreads, 0, b->stream>>>(ntotal, p.uidx);
	B_CUDA(cudaGetLastError());
	B_CUDA(cudaStreamSynchronize(b->stream));
	b->loaded = true;
	b->prepared = false;
	return MDGPU_OK;
}

int mdgpu_batch_get_particles(mdgpu_batch* h, int64_t ntotal, uint64_t* id, int32_t* cid, double* r, double* v,
                              double* F) {
	if (!h) return MDGPU_ERR_ARG;
	Batch* b = &h->b;
	if (ntotal != b->ntotal) return bfail(b, MDGPU_ERR_ARG, "ntotal must equal the sum of the box counts");
	if (!b->loaded) return bfail(b, MDGPU_ERR_STATE, "no molecules loaded");
	B_CUDA(cudaSetDevice(b->device));
	const Particles& p = b->buf[b->cur];
	struct {
		double* out;
		double *x, *y, *z;
	} sets[3] = {{r, p.rx, p.ry, p.rz}, {v, p.vx, p.vy, p.vz}, {F, p.fx, p.fy, p.fz}};
	for (auto& s : sets) {
		if (!s.out) continue;
		k_store3<<<blocks(ntotal), kThreads, 0, b->stream>>>(ntotal, s.x, s.y, s.z, p.uidx, b->stage);
		B_CUDA(cudaMemcpyAsync(s.out, b->stage, sizeof(double) * 3 * ntotal, cudaMemcpyDeviceToHost, b->stream));
		B_CUDA(cudaStreamSynchronize(b->stream));
	}
	if (id) {
		k_store1<uint64_t><<<blocks(ntotal), kThreads, 0, b->stream>>>(ntotal, p.id, p.uidx, (uint64_t*) b->stage);
		B_CUDA(cudaMemcpyAsync(id, b->stage, sizeof(uint64_t) * ntotal, cudaMemcpyDeviceToHost, b->stream));
		B_CUDA(cudaStreamSynchronize(b->stream));
	}
	if (cid) {
		k_store1<int32_t><<<blocks(ntotal), kThreads, 0, b->stream>>>(ntotal, p.cid, p.uidx, (int32_t*) b->stage);
		B_CUDA(cudaMemcpyAsync(cid, b->stage, sizeof(int32_t) * ntotal, cudaMemcpyDeviceToHost, b->stream));
		B_CUDA(cudaStreamSynchronize(b->stream));
	}
	B_CUDA(cudaGetLastError());
	return MDGPU_OK;
}

int mdgpu_batch_prepare(mdgpu_batch* h, double* out) {
	if (!h) return MDGPU_ERR_ARG;
	Batch* b = &h->b;
	if (!b->loaded) return bfail(b, MDGPU_ERR_STATE, "no molecules loaded");
	B_CUDA(cudaSetDevice(b->device));
	Launch L;
	int st = plan(b, b->tiles, L);
	if (st) return st;
	B_CUDA(launch_step(b, L, args(b, L, b->cur, 0, 0.0, b->prep)));
	b->cur = 1 - b->cur;
	st = check_status(b);
	if (st) return st;
	if (out) {
		B_CUDA(cudaMemcpy(out, b->prep, sizeof(double) * 4 * b->nboxes, cudaMemcpyDeviceToHost));
	}
	b->prepared = true;
	return MDGPU_OK;
}

int mdgpu_batch_run(mdgpu_batch* h, int32_t nsteps, double dt, double* per_step) {
	if (!h) return MDGPU_ERR_ARG;
	Batch* b = &h->b;
	if (!b->prepared) return bfail(b, MDGPU_ERR_STATE, "call mdgpu_batch_prepare first");
	if (nsteps < 0) return bfail(b, MDGPU_ERR_ARG, "nsteps must be >= 0");
	if (nsteps == 0) return MDGPU_OK;
	B_CUDA(cudaSetDevice(b->device));
	int st = run_steps(b, nsteps, dt);
	if (st) return st;
	st = check_status(b);
	float ms = 0.f;
	if (cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess) b->last_ms = ms;
	if (st) return st;
	if (per_step)
		B_CUDA(cudaMemcpy(per_step, b->records, sizeof(double) * 4 * b->nboxes * nsteps, cudaMemcpyDeviceToHost));
	return MDGPU_OK;
}

int mdgpu_batch_set_tiles(mdgpu_batch* h, int32_t list_cap, int32_t ctas_per_sm, int32_t dynamic) {
	if (!h) return MDGPU_ERR_ARG;
	Batch* b = &h->b;
	if (list_cap != 32 && list_cap != 64) return bfail(b, MDGPU_ERR_ARG, "list_cap must be 32 or 64");
	if (ctas_per_sm != 1 && ctas_per_sm != 2) return bfail(b, MDGPU_ERR_ARG, "ctas_per_sm must be 1 or 2");
	if (dynamic != 0 && dynamic != 1) return bfail(b, MDGPU_ERR_ARG, "dynamic must be 0 or 1");
	if (ctas_per_sm == 2 && b->max_bin_bytes > 110 * 1024)
		return bfail(b, MDGPU_ERR_CAPACITY, "the largest box needs one CTA per SM");
	b->tiles.cap = list_cap;
	b->tiles.ctas = ctas_per_sm;
	b->tiles.dynamic = dynamic;
	return MDGPU_OK;
}

int mdgpu_batch_get_tiles(const mdgpu_batch* h, int32_t tiles[3]) {
	if (!h || !tiles) return MDGPU_ERR_ARG;
	tiles[0] = h->b.tiles.cap;
	tiles[1] = h->b.tiles.ctas;
	tiles[2] = h->b.tiles.dynamic;
	return MDGPU_OK;
}

int mdgpu_batch_autotune(mdgpu_batch* h, double dt, int32_t trial_steps, int32_t best[3], double* ms) {
	if (!h) return MDGPU_ERR_ARG;
	Batch* b = &h->b;
	if (!b->prepared) return bfail(b, MDGPU_ERR_STATE, "call mdgpu_batch_prepare first");
	if (trial_steps < 1) return bfail(b, MDGPU_ERR_ARG, "trial_steps must be >= 1");
	B_CUDA(cudaSetDevice(b->device));
	if (!b->backup_alloc) {
		B_CUDA(alloc_particles(b->backup, b->ntotal));
		b->backup_alloc = true;
	}
	const int cur0 = b->cur;
	B_CUDA(copy_particles(b->backup, b->buf[cur0], b->ntotal, b->stream));
	const Tiles keep = b->tiles;
	Tiles bestt = keep;
	double bestms = 1e300;
	int k = 0;
	for (int cap : {32, 64})
		for (int ctas : {1, 2})
			for (int dyn : {0, 1}) {
				double t = -1.0;
				if (!(ctas == 2 && b->max_bin_bytes > 110 * 1024)) {
					b->tiles = Tiles{cap, ctas, dyn};
					// warm-up (graph capture), then the timed replay, each from the saved state
					int st = MDGPU_OK;
					double best_rep = 1e300;
					for (int rep = 0; rep < 2 && st == MDGPU_OK; rep++) {
						b->cur = cur0;
						st = run_steps(b, trial_steps, dt);
						if (st == MDGPU_OK) st = check_status(b);
						if (st == MDGPU_OK) {
							float f = 0.f;
							B_CUDA(cudaEventElapsedTime(&f, b->ev0, b->ev1));
							if (rep > 0) best_rep = f;
						}
						B_CUDA(copy_particles(b->buf[cur0], b->backup, b->ntotal, b->stream));
					}
					if (st != MDGPU_OK) {
						b->tiles = keep;
						b->cur = cur0;
						return st;
					}
					t = best_rep / trial_steps;
					if (t < bestms) {
						bestms = t;
						bestt = b->tiles;
					}
				}
				if (ms) ms[k] = t;
				k++;
			}
	B_CUDA(cudaStreamSynchronize(b->stream));
	b->cur = cur0;
	b->tiles = bestt;
	if (best) {
		best[0] = bestt.cap;
		best[1] = bestt.ctas;
		best[2] = bestt.dynamic;
	}
	return MDGPU_OK;
}

int mdgpu_batch_last_run_ms(const mdgpu_batch* h, double* ms) {
	if (!h || !ms) return MDGPU_ERR_ARG;
	*ms = h->b.last_ms;
	return MDGPU_OK;
}

int mdgpu_batch_set_barrier_timeout(mdgpu_batch* h, int64_t ns) {
	if (!h) return MDGPU_ERR_ARG;
	Batch* b = &h->b;
	if (ns < 0) return bfail(b, MDGPU_ERR_ARG, "timeout must be >= 0");
	b->timeout_ns = ns;
	for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);   // the limit is a kernel argument
	b->graphs.clear();
	return MDGPU_OK;
}

}  // extern "C"
