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
	// Verlet-skin mode: the state stays in src (dst is the sort scratch); a box is re-binned and its
	// lists rebuilt when one of its molecules moved more than skin/2 since its last build
	int skin;
	double half_skin2;
	brick::Lists lists;
	int* box_flag;              // nboxes: 1 = built in this step
	int* valid;                 // 0: every box builds (molecules just loaded)
	int build_cap;              // staged capacity of the list build
	brick::Const lc;            // constants of the list evaluation (its staged capacity)
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
	const Particles& P = a.skin ? a.src : a.dst;
	double mv2 = 0.0;
	bool bad = false;
	for (int t = tid; t < B.n; t += kThreads) {
		const int64_t i = B.poff + t;
		const int ty = P.cid[i];
		double vx = P.vx[i], vy = P.vy[i], vz = P.vz[i];
		if (a.integrate) {
			const double k = a.kick.post[ty];
			vx = __dadd_rn(vx, __dmul_rn(k, P.fx[i]));
			vy = __dadd_rn(vy, __dmul_rn(k, P.fy[i]));
			vz = __dadd_rn(vz, __dmul_rn(k, P.fz[i]));
			P.vx[i] = vx;
			P.vy[i] = vy;
			P.vz[i] = vz;
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

// Phase A of the Verlet-skin mode for box b: kick-drift in place (no wrap), displacement against
// the positions of the box's last build; when one moved more than skin/2 (or the lists are not
// valid) the box is wrapped, binned and sorted into the scratch buffer and copied back.
__device__ void skin_box(const StepArgs& a, const BatchBox& B, int b, unsigned char* smem) {
	__shared__ int s_any;
	const int tid = threadIdx.x;
	if (tid == 0) s_any = 0;
	__syncthreads();
	if (a.integrate) {
		bool moved = false;
		for (int t = tid; t < B.n; t += kThreads) {
			const int64_t i = B.poff + t;
			const double k = a.kick.pre[a.src.cid[i]];
			const double vx0 = a.src.vx[i], vy0 = a.src.vy[i], vz0 = a.src.vz[i];
			const double fx = a.src.fx[i], fy = a.src.fy[i], fz = a.src.fz[i];
			const double x0 = a.src.rx[i], y0 = a.src.ry[i], z0 = a.src.rz[i];
			const double vx = __dadd_rn(__dmul_rn(1.0, vx0), __dmul_rn(k, fx));
			const double vy = __dadd_rn(__dmul_rn(1.0, vy0), __dmul_rn(k, fy));
			const double vz = __dadd_rn(__dmul_rn(1.0, vz0), __dmul_rn(k, fz));
			const double x = __dadd_rn(x0, __dmul_rn(a.dt, vx));
			const double y = __dadd_rn(y0, __dmul_rn(a.dt, vy));
			const double z = __dadd_rn(z0, __dmul_rn(a.dt, vz));
			a.src.vx[i] = vx;
			a.src.vy[i] = vy;
			a.src.vz[i] = vz;
			a.src.rx[i] = x;
			a.src.ry[i] = y;
			a.src.rz[i] = z;
			const double dx = x - a.lists.rx_ref[i], dy = y - a.lists.ry_ref[i], dz = z - a.lists.rz_ref[i];
			if (!(dx * dx + dy * dy + dz * dz <= a.half_skin2)) moved = true;
		}
		if (moved) s_any = 1;
	}
	__syncthreads();
	const bool rebuild = s_any != 0 || *a.valid == 0;
	if (rebuild) {
		StepArgs a2 = a;
		a2.integrate = 0;
		bin_box(a2, B, smem);
		for (int t = tid; t < B.n; t += kThreads) {
			const int64_t i = B.poff + t;
			a.src.rx[i] = a.dst.rx[i];
			a.src.ry[i] = a.dst.ry[i];
			a.src.rz[i] = a.dst.rz[i];
			a.src.vx[i] = a.dst.vx[i];
			a.src.vy[i] = a.dst.vy[i];
			a.src.vz[i] = a.dst.vz[i];
			a.src.id[i] = a.dst.id[i];
			a.src.cid[i] = a.dst.cid[i];
			a.src.uidx[i] = a.dst.uidx[i];
		}
	}
	if (tid == 0) a.box_flag[b] = rebuild ? 1 : 0;
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
__global__ void __launch_bounds__(kThreads, 2) k_batch_step(StepArgs a) {
	extern __shared__ __align__(16) unsigned char smem[];
	__shared__ int s_flag;
	__shared__ int s_item;
	if (threadIdx.x == 0) s_flag = (*((volatile int*) a.status) & kStatusTimeout) ? 1 : 0;
	__syncthreads();
	if (s_flag) return;   // an earlier launch gave up at a barrier: do nothing until the host resets

	// ---- A: per box kick-drift, wrap, bin, sort ----------------------------------------------
	if (a.skin)
		for_my_boxes(a, [&](int b) { skin_box(a, a.boxes[b], b, smem); });
	else
		for_my_boxes(a, [&](int b) { bin_box(a, a.boxes[b], smem); });
	if (!grid_barrier(a.bar, a.status, a.timeout_ns, &s_flag)) return;

	// brick of a global brick index: box with brick0[box] <= item < brick0[box + 1]
	auto box_of = [&](int item) {
		int lo = 0, hi = a.nboxes - 1;
		while (lo < hi) {
			const int mid = (lo + hi + 1) >> 1;
			if (a.brick0[mid] <= item)
				lo = mid;
			else
				hi = mid - 1;
		}
		return lo;
	};
	// every brick once, by static stride or from the queue bar[q]
	auto for_bricks = [&](int q, auto&& f) {
		if (a.dynamic) {
			for (;;) {
				if (threadIdx.x == 0) s_item = (int) atomicAdd(a.bar + q, 1u);
				__syncthreads();
				const int item = s_item;
				__syncthreads();
				if (item >= a.total_bricks) break;
				f(item);
			}
		} else {
			for (int item = blockIdx.x; item < a.total_bricks; item += gridDim.x) f(item);
		}
	};

	if (!a.skin) {
		// ---- B: pair forces of every brick (filter and evaluation) ----------------------------
		const brick::SmemLayout L = brick::layout(a.pc.s_cap, kFP64, kCap);
		brick::load_params(smem, L, a.pp, a.pc.ns);
		__syncthreads();
		for_bricks(2, [&](int item) {
			const BatchBox& B = a.boxes[box_of(item)];
			brick::pairs<kFP64, kSingle, kLjIsRc, kCap, false>(a.pc, B.bx, item - B.brick0, item, smem, a.dst.rx, a.dst.ry,
			                                            a.dst.rz, a.dst.cid, a.cstart, a.dst.fx, a.dst.fy, a.dst.fz,
			                                            a.partials, a.status);
			__syncthreads();
		});
	} else {
		// ---- B1: candidate lists of the boxes that were re-binned -----------------------------
		for_bricks(2, [&](int item) {
			const int b = box_of(item);
			if (!a.box_flag[b]) return;
			const BatchBox& B = a.boxes[b];
			brick::build_lists(B.bx, item - B.brick0, a.build_cap, smem, a.src.rx, a.src.ry, a.src.rz, a.cstart, a.lists,
			                   item);
			__syncthreads();
		});
		if (!grid_barrier(a.bar, a.status, a.timeout_ns, &s_flag)) return;
		// ---- B2: list evaluation of every brick -----------------------------------------------
		const brick::SmemLayout L = brick::layout(a.lc.s_cap, kFP64, 0, false);
		brick::load_params(smem, L, a.pp, a.lc.ns);
		if (threadIdx.x == 0)
			reinterpret_cast<float4*>(smem + L.hi)[a.lc.s_cap] =
			    make_float4(1e15f, 1e15f, 1e15f, __uint_as_float((256u << 18) | (256u << 9) | 256u));
		__syncthreads();
		for_bricks(3, [&](int item) {
			const BatchBox& B = a.boxes[box_of(item)];
			brick::list_pairs<kFP64, kSingle, kLjIsRc, false>(a.lc, B.bx, item - B.brick0, item, smem, a.src.rx, a.src.ry,
			                                           a.src.rz, a.src.cid, a.cstart, a.src.fx, a.src.fy, a.src.fz,
			                                           a.partials, a.status, a.lists, brick::Kick{});
			__syncthreads();
		});
	}
	if (!grid_barrier(a.bar, a.status, a.timeout_ns, &s_flag)) return;

	// ---- C: per box post-kick and records ----------------------------------------------------
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		a.bar[2] = 0u;   // queues are idle until the next launch
		a.bar[3] = 0u;
		if (a.skin) *a.valid = 1;
	}
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

// positions -> caller order, wrapped into [0, L) of their box (r<0 -> r+L, r>=L -> r-L)
__global__ void k_store3_wrap(int64_t n, const double* x, const double* y, const double* z, const int32_t* uidx,
                              const int32_t* bid, const double* len, double* __restrict__ aos) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const int64_t u = uidx[s];
	const double* L = len + 3 * bid[s];
	const double r[3] = {x[s], y[s], z[s]};
	for (int d = 0; d < 3; d++) {
		double w = r[d];
		if (w < 0.0)
			w = __dadd_rn(w, L[d]);
		else if (w >= L[d])
			w = __dsub_rn(w, L[d]);
		aos[3 * u + d] = w;
	}
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
	std::vector<int32_t> h_brick0;
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
	// Verlet-skin mode
	double skin = 0.0;
	std::vector<double> h_len;    // nboxes x 3
	std::vector<int64_t> h_count;
	int list_cap = 0;
	unsigned short* nbr = nullptr;
	unsigned short* nbr_count = nullptr;
	double* r_ref = nullptr;
	int* box_flag = nullptr;
	int* valid = nullptr;
	unsigned char* kind = nullptr;
	unsigned long long* builds = nullptr;
	int32_t* d_bid = nullptr;     // box of each molecule slot
	double* d_len = nullptr;      // nboxes x 3
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
	brick::Const lc;   // list evaluation (skin mode)
	int build_cap;     // list build staging capacity (skin mode)
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
	if (b->skin > 0.0) {
		const int lcap = brick::capacity_for(budget, fp64, 0, false);
		L.lc = brick::make_const(b->sp.n, lcap, b->rc, b->rc_lj);
		int bcap = 256;
		while (brick::build_bytes(bcap + 64) <= budget) bcap += 64;
		L.build_cap = bcap;
		L.smem = std::max({brick::layout(lcap, fp64, 0, false).total, brick::build_bytes(bcap), b->max_bin_bytes});
	}
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
	if (b->skin > 0.0) {
		a.skin = 1;
		a.half_skin2 = 0.25 * b->skin * b->skin;
		a.lists.nbr = b->nbr;
		a.lists.count = b->nbr_count;
		a.lists.rx_ref = b->r_ref;
		a.lists.ry_ref = b->r_ref + b->ntotal;
		a.lists.rz_ref = b->r_ref + 2 * b->ntotal;
		a.lists.n = b->ntotal;
		a.lists.cap = b->list_cap;
		a.lists.builds = b->builds;
		a.lists.sentinel = L.lc.s_cap;
		a.lists.kind = b->kind;
		a.box_flag = b->box_flag;
		a.valid = b->valid;
		a.build_cap = L.build_cap;
		a.lc = L.lc;
	}
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
			if (b->skin == 0.0) src = 1 - src;   // the skin mode keeps the state in one buffer
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
	if ((nsteps & 1) && b->skin == 0.0) b->cur = 1 - b->cur;
	return MDGPU_OK;
}

// The per-box table (grids on cells of edge >= cutoff, or >= cutoff + skin in the skin mode) and the
// offsets of every box's molecules, cells and bricks; host side only.
int box_table(Batch* b) {
	const int nboxes = b->nboxes;
	const double grid_rc = b->rc + b->skin;
	b->h_boxes.assign(nboxes, BatchBox{});
	b->h_brick0.assign(nboxes + 1, 0);
	b->max_bin_bytes = 0;
	int64_t poff = 0, coff = 0, brick0 = 0;
	for (int k = 0; k < nboxes; k++) {
		if (b->h_count[k] < 1) return bfail(b, MDGPU_ERR_ARG, "every box needs at least one molecule");
		Grid g{};
		int st = setup_grid(b->h_len.data() + 3 * k, grid_rc, 1.0, g, b->err);
		if (st) {
			b->err = "box " + std::to_string(k) + ": " + b->err;
			return st;
		}
		if (b->skin > 0.0) even_grid(g);
		if (g.ncells > 65535) return bfail(b, MDGPU_ERR_CAPACITY, "box " + std::to_string(k) + " has more than 65535 cells");
		if (b->h_count[k] > 65535)
			return bfail(b, MDGPU_ERR_CAPACITY, "box " + std::to_string(k) + " has more than 65535 molecules");
		BatchBox& B = b->h_boxes[k];
		brick::init_box(B.bx, g, grid_rc, (int32_t) coff, 0.5 * b->skin);
		B.poff = poff;
		B.n = (int32_t) b->h_count[k];
		B.brick0 = (int32_t) brick0;
		b->h_brick0[k] = (int32_t) brick0;
		b->max_bin_bytes = std::max(b->max_bin_bytes, bin_bytes(b->h_count[k], g.ncells));
		poff += b->h_count[k];
		coff += g.ncells;
		brick0 += (int64_t) B.bx.nb[0] * B.bx.nb[1] * B.bx.nb[2];
		if (poff >= (1LL << 28) || coff >= (1LL << 30) || brick0 >= (1LL << 30))
			return bfail(b, MDGPU_ERR_CAPACITY, "the batch exceeds 2^28 molecules or 2^30 cells/bricks");
	}
	b->h_brick0[nboxes] = (int32_t) brick0;
	b->ntotal = poff;
	b->total_cells = (int) coff;
	b->total_bricks = (int) brick0;
	b->h_order.resize(nboxes);
	for (int k = 0; k < nboxes; k++) b->h_order[k] = k;
	std::stable_sort(b->h_order.begin(), b->h_order.end(),
	                 [&](int x, int y) { return b->h_boxes[x].n > b->h_boxes[y].n; });
	return MDGPU_OK;
}

// Device copies of the box table and the buffers sized by it (again after a change of the skin).
int upload_table(Batch* b) {
	void* old[] = {b->cstart, b->partials, b->d_boxes, b->d_brick0, b->d_order, b->kind};
	for (void* x : old) cudaFree(x);
	b->cstart = nullptr;
	b->partials = nullptr;
	b->d_boxes = nullptr;
	b->d_brick0 = nullptr;
	b->d_order = nullptr;
	b->kind = nullptr;
	for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);
	b->graphs.clear();
	const int nboxes = b->nboxes;
	B_CUDA(cudaMalloc(&b->cstart, sizeof(int32_t) * (b->total_cells + 1)));
	B_CUDA(cudaMalloc(&b->partials, sizeof(double) * 4 * b->total_bricks));
	B_CUDA(cudaMalloc(&b->kind, b->total_bricks));
	B_CUDA(cudaMalloc(&b->d_boxes, sizeof(BatchBox) * nboxes));
	B_CUDA(cudaMemcpy(b->d_boxes, b->h_boxes.data(), sizeof(BatchBox) * nboxes, cudaMemcpyHostToDevice));
	B_CUDA(cudaMalloc(&b->d_brick0, sizeof(int32_t) * (nboxes + 1)));
	B_CUDA(cudaMemcpy(b->d_brick0, b->h_brick0.data(), sizeof(int32_t) * (nboxes + 1), cudaMemcpyHostToDevice));
	B_CUDA(cudaMalloc(&b->d_order, sizeof(int32_t) * nboxes));
	B_CUDA(cudaMemcpy(b->d_order, b->h_order.data(), sizeof(int32_t) * nboxes, cudaMemcpyHostToDevice));
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
	if (!(lj_cutoff >= 0)) return bfail(b, MDGPU_ERR_ARG, "lj_cutoff must be 0 (= cutoff) or positive");
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
	b->h_len.assign(lengths, lengths + 3 * (size_t) nboxes);
	b->h_count.assign(counts, counts + nboxes);
	st = box_table(b);
	if (st) return st;

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
	st = upload_table(b);
	if (st) return st;
	B_CUDA(cudaMalloc(&b->prep, sizeof(double) * 4 * nboxes));
	B_CUDA(cudaMalloc(&b->status, sizeof(int)));
	B_CUDA(cudaMemset(b->status, 0, sizeof(int)));
	B_CUDA(cudaMallocHost(&b->h_status, sizeof(int)));
	B_CUDA(cudaMalloc(&b->bar, sizeof(unsigned) * 4));
	B_CUDA(cudaMemset(b->bar, 0, sizeof(unsigned) * 4));
	PairParams hp = pair_params(b->sp, b->rc, b->rc_lj);
	B_CUDA(cudaMalloc(&b->d_pp, sizeof(PairParams)));
	B_CUDA(cudaMemcpy(b->d_pp, &hp, sizeof(PairParams), cudaMemcpyHostToDevice));
	// box of each molecule slot and the box lengths (positions are wrapped on output)
	{
		std::vector<int32_t> bid(b->ntotal);
		for (int k = 0; k < nboxes; k++)
			for (int64_t i = 0; i < b->h_count[k]; i++) bid[b->h_boxes[k].poff + i] = k;
		B_CUDA(cudaMalloc(&b->d_bid, sizeof(int32_t) * b->ntotal));
		B_CUDA(cudaMemcpy(b->d_bid, bid.data(), sizeof(int32_t) * b->ntotal, cudaMemcpyHostToDevice));
		B_CUDA(cudaMalloc(&b->d_len, sizeof(double) * 3 * nboxes));
		B_CUDA(cudaMemcpy(b->d_len, b->h_len.data(), sizeof(double) * 3 * nboxes, cudaMemcpyHostToDevice));
	}
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
	                b->d_brick0, b->d_order, b->stage, b->nbr, b->nbr_count, b->r_ref, b->box_flag,
	                b->valid, b->kind, b->builds, b->d_bid, b->d_len};
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
	if (b->valid) B_CUDA(cudaMemsetAsync(b->valid, 0, sizeof(int), b->stream));
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
		if (s.out == r)
			k_store3_wrap<<<blocks(ntotal), kThreads, 0, b->stream>>>(ntotal, s.x, s.y, s.z, p.uidx, b->d_bid, b->d_len,
			                                                          b->stage);
		else
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
	if (b->skin == 0.0) b->cur = 1 - b->cur;
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
	// In the Verlet-skin mode the lists live in global memory and the shared-memory layout does not
	// depend on the list depth (both depths compile to the same register count), so only the current
	// depth is timed there and the other depth's candidates report -1.
	const bool skin_mode = b->skin > 0.0;
	for (int cap : {32, 64})
		for (int ctas : {1, 2})
			for (int dyn : {0, 1}) {
				double t = -1.0;
				if (!(ctas == 2 && b->max_bin_bytes > 110 * 1024) && !(skin_mode && cap != keep.cap)) {
					b->tiles = Tiles{cap, ctas, dyn};
					// warm-up (graph capture), then the timed replay, each from the saved state
					int st = MDGPU_OK;
					double best_rep = 1e300;
					for (int rep = 0; rep < 2 && st == MDGPU_OK; rep++) {
						b->cur = cur0;
						if (b->valid) B_CUDA(cudaMemsetAsync(b->valid, 0, sizeof(int), b->stream));
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
	if (b->valid) B_CUDA(cudaMemsetAsync(b->valid, 0, sizeof(int), b->stream));
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

int mdgpu_batch_set_skin(mdgpu_batch* h, double skin) {
	if (!h) return MDGPU_ERR_ARG;
	Batch* b = &h->b;
	if (!(skin >= 0.0) || !(skin < b->rc)) return bfail(b, MDGPU_ERR_ARG, "skin must be in [0, cutoff)");
	B_CUDA(cudaSetDevice(b->device));
	B_CUDA(cudaStreamSynchronize(b->stream));
	const double old = b->skin;
	b->skin = skin;
	int st = box_table(b);
	if (!st) st = upload_table(b);
	if (st) {
		b->skin = old;
		box_table(b);
		upload_table(b);
		return st;
	}
	if (b->max_bin_bytes > 110 * 1024) b->tiles.ctas = 1;
	void* lists[] = {b->nbr, b->nbr_count, b->r_ref, b->box_flag, b->valid, b->builds};
	for (void* x : lists) cudaFree(x);
	b->nbr = b->nbr_count = nullptr;
	b->r_ref = nullptr;
	b->box_flag = b->valid = nullptr;
	b->builds = nullptr;
	if (skin > 0.0) {
		// list capacity from the densest box (x 1.5 for local fluctuations)
		double rho = 0.0;
		for (int k = 0; k < b->nboxes; k++)
			rho = std::max(rho, b->h_count[k] / (b->h_len[3 * k] * b->h_len[3 * k + 1] * b->h_len[3 * k + 2]));
		const double rl = b->rc + skin;
		int cap = (int) std::ceil(1.25 * 4.18879020478639 * rl * rl * rl * rho * 1.5) + 32;
		cap = std::min((cap + 31) & ~31, 65504);
		b->list_cap = cap;
		B_CUDA(cudaMalloc(&b->nbr, sizeof(unsigned short) * (size_t) cap * b->ntotal));
		B_CUDA(cudaMalloc(&b->nbr_count, sizeof(unsigned short) * b->ntotal));
		B_CUDA(cudaMalloc(&b->r_ref, sizeof(double) * 3 * b->ntotal));
		B_CUDA(cudaMalloc(&b->box_flag, sizeof(int) * b->nboxes));
		B_CUDA(cudaMalloc(&b->valid, sizeof(int)));
		B_CUDA(cudaMemset(b->valid, 0, sizeof(int)));
		B_CUDA(cudaMalloc(&b->builds, sizeof(unsigned long long)));
		B_CUDA(cudaMemset(b->builds, 0, sizeof(unsigned long long)));
	}
	b->prepared = false;
	return MDGPU_OK;
}

int mdgpu_batch_skin_builds(const mdgpu_batch* h, int64_t* builds) {
	if (!h || !builds) return MDGPU_ERR_ARG;
	const Batch* b = &h->b;
	*builds = 0;
	if (!b->builds) return MDGPU_OK;
	unsigned long long v = 0;
	if (cudaMemcpy(&v, b->builds, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return MDGPU_ERR_CUDA;
	*builds = (int64_t) v;
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
