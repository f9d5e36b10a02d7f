// Linked-cell binning by counting sort into a cell-ordered structure of arrays.
//
// Per update (LinkedCells::update, particleContainer/LinkedCells.cpp:165-180, paths relative to
// madpac/mardyn/):
//   1. bin:        periodic wrap of each coordinate (r<0 -> r+L, r>=L -> r-L: the position of the
//                  halo image that survives DomainDecompDummy::exchangeMolecules +
//                  LinkedCells::deleteOuterParticles, parallel/DomainDecompDummy.cpp:64-70, 93-99,
//                  LinkedCells.cpp:356-369), the cell coordinate floor((r - haloMin)/cellLength)
//                  in IEEE double with no contraction (LinkedCells.cpp:543), and an atomic
//                  arrival rank per cell.
//   2. scan:       exclusive prefix sum of the cell counts.
//   3. scatter:    slot = cell_start + rank (arrival order, not deterministic).
//   4. cell sort:  one warp per cell orders its molecules by id and gathers every field into
//                  the other buffer, so the final order (cell, id) does not depend on timing.
// launch_bin runs these as separate kernels (the drop-in update). launch_rebuild runs them as one
// cooperative kernel with bounded grid barriers that returns at once unless the Verlet-skin mode
// asked for a build in this step.
#include <cuda_runtime.h>

#include <mutex>

#include <algorithm>

#include "grid_sync.cuh"
#include "md_internal.h"

namespace mdgpu {
namespace {

constexpr int kScanBlock = 1024;   // elements per scan block (256 threads x 4)

// Wrap the position r in place and return its inner cell; flags positions outside the halo box.
__device__ __forceinline__ int32_t wrap_cell(double r[3], const Grid& g, bool& bad) {
	int ci[3];
	for (int d = 0; d < 3; d++) {
		double x = r[d];
		double xw = x;
		if (x < 0.0)
			xw = __dadd_rn(x, g.L[d]);
		else if (x >= g.L[d])
			xw = __dsub_rn(x, g.L[d]);
		r[d] = xw;
		int c = (int) floor(__ddiv_rn(__dsub_rn(xw, g.halo_min[d]), g.cell_length[d]));
		// inner cells are 1..nc in the halo-inclusive numbering
		if (c < 1 || c > g.nc[d]) {
			bad = true;
			c = c < 1 ? 1 : g.nc[d];
		}
		ci[d] = c - 1;
		if (!(x == x)) bad = true;
	}
	return (int32_t) (((int64_t) ci[2] * g.nc[1] + ci[1]) * g.nc[0] + ci[0]);
}

// Wrap molecule i, return its inner cell and flag positions outside the halo box.
__device__ __forceinline__ int32_t bin_one(int64_t i, double* rx, double* ry, double* rz, const Grid& g, bool& bad) {
	const double r0[3] = {rx[i], ry[i], rz[i]};
	double r[3] = {r0[0], r0[1], r0[2]};
	const int32_t c = wrap_cell(r, g, bad);
	if (r[0] != r0[0]) rx[i] = r[0];
	if (r[1] != r0[1]) ry[i] = r[1];
	if (r[2] != r0[2]) rz[i] = r[2];
	return c;
}

__device__ __forceinline__ bool key_less(uint64_t ka, int32_t sa, uint64_t kb, int32_t sb) {
	return ka < kb || (ka == kb && sa < sb);
}

// Molecule `from` to slot `to` of the other buffer. Every field is loaded before the first store:
// the compiler cannot tell the two buffers apart, and a load after a store to a possibly aliasing
// address would wait for it, serialising the loads' latencies.
__device__ __forceinline__ void move_one(int32_t from, int32_t to, uint64_t key, int64_t c, const Particles& src,
                                         const Particles& dst, int32_t* cell_out, bool with_forces) {
	const double x = src.rx[from], y = src.ry[from], z = src.rz[from];
	const double vx = src.vx[from], vy = src.vy[from], vz = src.vz[from];
	double fx = 0.0, fy = 0.0, fz = 0.0;
	if (with_forces) {
		fx = src.fx[from];
		fy = src.fy[from];
		fz = src.fz[from];
	}
	const int32_t ci = src.cid[from], ui = src.uidx[from];
	dst.rx[to] = x;
	dst.ry[to] = y;
	dst.rz[to] = z;
	dst.vx[to] = vx;
	dst.vy[to] = vy;
	dst.vz[to] = vz;
	if (with_forces) {
		dst.fx[to] = fx;
		dst.fy[to] = fy;
		dst.fz[to] = fz;
	}
	dst.id[to] = key;
	dst.cid[to] = ci;
	dst.uidx[to] = ui;
	cell_out[to] = (int32_t) c;
}

// Cells of up to 32 x kSortRegs molecules are ranked from keys held in registers (warp shuffles);
// larger ones read the keys from global memory.
constexpr int kSortRegs = 4;

// One warp per cell c: order the cell's molecules by (id, previous slot) and gather all fields.
// Each molecule's slot is the number of the cell's molecules with a smaller key.
__device__ __forceinline__ void sort_cell(int64_t c, int lane, const int32_t* start, const int32_t* perm,
                                          const Particles& src, const Particles& dst, int32_t* cell_out,
                                          bool with_forces) {
	const int32_t s = start[c], m = start[c + 1] - s;
	if (m <= 32 * kSortRegs) {
		uint64_t key[kSortRegs];
		int32_t from[kSortRegs], pos[kSortRegs];
#pragma unroll
		for (int r = 0; r < kSortRegs; r++) {
			const int32_t e = 32 * r + lane;
			from[r] = 0x7fffffff;   // padding sorts after every molecule
			key[r] = ~0ull;
			pos[r] = 0;
			if (e < m) {
				from[r] = perm[s + e];
				key[r] = src.id[from[r]];
			}
		}
#pragma unroll
		for (int r2 = 0; r2 < kSortRegs; r2++) {
			if (32 * r2 >= m) break;
			for (int k = 0; k < 32; k++) {
				const uint64_t ok = __shfl_sync(0xffffffffu, key[r2], k);
				const int32_t of = __shfl_sync(0xffffffffu, from[r2], k);
#pragma unroll
				for (int r = 0; r < kSortRegs; r++)
					if (key_less(ok, of, key[r], from[r])) pos[r]++;
			}
		}
#pragma unroll
		for (int r = 0; r < kSortRegs; r++)
			if (32 * r + lane < m) move_one(from[r], s + pos[r], key[r], c, src, dst, cell_out, with_forces);
		return;
	}
	for (int32_t e0 = 0; e0 < m; e0 += 32) {
		const int32_t e = e0 + lane;
		if (e >= m) continue;
		const int32_t from = perm[s + e];
		const uint64_t key = src.id[from];
		int32_t pos = 0;
		for (int32_t k = 0; k < m; k++) {
			const int32_t of = perm[s + k];
			if (key_less(src.id[of], of, key, from)) pos++;
		}
		move_one(from, s + pos, key, c, src, dst, cell_out, with_forces);
	}
}

__global__ void k_bin_cells(int64_t n, double* __restrict__ rx, double* __restrict__ ry, double* __restrict__ rz,
                            Grid g, int32_t* __restrict__ cell, int32_t* __restrict__ rank,
                            int32_t* __restrict__ count, int* status) {
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	bool bad = false;
	const int32_t c = bin_one(i, rx, ry, rz, g, bad);
	if (bad) atomicOr(status, kStatusOutsideHalo);
	cell[i] = c;
	rank[i] = atomicAdd(&count[c], 1);
}

// Block-local exclusive scan of kScanBlock counts; block totals go to sums.
__global__ void k_scan_local(int64_t n, const int32_t* __restrict__ in, int32_t* __restrict__ out,
                             int32_t* __restrict__ sums) {
	__shared__ int32_t warp_tot[8];
	int64_t base = (int64_t) blockIdx.x * kScanBlock + threadIdx.x * 4;
	int32_t v[4];
	int32_t t = 0;
	for (int k = 0; k < 4; k++) {
		v[k] = (base + k < n) ? in[base + k] : 0;
		t += v[k];
	}
	int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int32_t inc = t;
	for (int o = 1; o < 32; o <<= 1) {
		int32_t y = __shfl_up_sync(0xffffffffu, inc, o);
		if (lane >= o) inc += y;
	}
	if (lane == 31) warp_tot[warp] = inc;
	__syncthreads();
	if (warp == 0) {
		int32_t w = lane < 8 ? warp_tot[lane] : 0;
		for (int o = 1; o < 8; o <<= 1) {
			int32_t y = __shfl_up_sync(0xffffffffu, w, o);
			if (lane >= o) w += y;
		}
		if (lane < 8) warp_tot[lane] = w;
	}
	__syncthreads();
	int32_t excl = inc - t + (warp > 0 ? warp_tot[warp - 1] : 0);
	for (int k = 0; k < 4; k++) {
		if (base + k < n) out[base + k] = excl;
		excl += v[k];
	}
	if (threadIdx.x == blockDim.x - 1) sums[blockIdx.x] = excl;
}

// Exclusive block scan of one value per thread (blockDim.x a multiple of 32, <= 1024): the
// thread's exclusive prefix, the block total in *total. Every thread of the block must call it.
__device__ __forceinline__ int32_t block_excl_scan(int32_t v, int32_t* total) {
	__shared__ int32_t wt[32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (int) (blockDim.x >> 5);
	int32_t inc = v;
	for (int o = 1; o < 32; o <<= 1) {
		int32_t y = __shfl_up_sync(0xffffffffu, inc, o);
		if (lane >= o) inc += y;
	}
	if (lane == 31) wt[warp] = inc;
	__syncthreads();
	if (warp == 0) {
		int32_t w = lane < nw ? wt[lane] : 0;
		for (int o = 1; o < 32; o <<= 1) {
			int32_t y = __shfl_up_sync(0xffffffffu, w, o);
			if (lane >= o) w += y;
		}
		wt[lane] = w;
	}
	__syncthreads();
	const int32_t excl = inc - v + (warp > 0 ? wt[warp - 1] : 0);
	*total = wt[nw - 1];
	__syncthreads();
	return excl;
}

// Single block: exclusive scan of the block totals, total appended at sums[nb].
__global__ void k_scan_sums(int64_t nb, int32_t* sums) {
	int32_t carry = 0;
	for (int64_t base = 0; base < nb; base += blockDim.x) {
		int64_t i = base + threadIdx.x;
		int32_t v = i < nb ? sums[i] : 0;
		int32_t tot;
		const int32_t excl = block_excl_scan(v, &tot);
		if (i < nb) sums[i] = carry + excl;
		carry += tot;
	}
	if (threadIdx.x == 0) sums[nb] = carry;
}

__global__ void k_scan_add(int64_t n, int32_t* __restrict__ out, const int32_t* __restrict__ sums, int64_t nb) {
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] += sums[i / kScanBlock];
	if (i == 0) out[n] = sums[nb];
}

__global__ void k_scatter(int64_t n, const int32_t* __restrict__ cell, const int32_t* __restrict__ rank,
                          const int32_t* __restrict__ start, int32_t* __restrict__ perm) {
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) perm[start[cell[i]] + rank[i]] = (int32_t) i;
}

__global__ void k_cell_sort(int64_t ncells, const int32_t* __restrict__ start, const int32_t* __restrict__ perm,
                            Particles src, Particles dst, int32_t* __restrict__ cell_out, bool with_forces) {
	int64_t c = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (c >= ncells) return;
	sort_cell(c, threadIdx.x & 31, start, perm, src, dst, cell_out, with_forces);
}

// ---- the whole rebuild in one cooperative launch ----------------------------------------------

struct RebuildArgs {
	int64_t n;
	Grid g;
	Particles p, q;
	int32_t *cell, *rank, *perm, *count, *start;
	int4* slot;                 // per arrival slot: cell, cell start, cell end, previous slot
	unsigned long long* look;   // per CTA: the scan's published value (flag in bits 62-63)
	int* status;
	const int* flag;
	int step;
	unsigned* bar;
	int64_t timeout_ns;
	unsigned* brick_counts;   // sparse/dense brick counts, zeroed for the list build that follows
	double* xs;               // nx more planes of n doubles sorted with the molecules (may be none)
	double* xt;               // nx planes of scratch for them
	int nx;
};

constexpr int kRebuildThreads = 256;
constexpr unsigned long long kLookAggregate = 1ull << 62;   // the CTA's own cell sum
constexpr unsigned long long kLookPrefix = 2ull << 62;      // the sum of every cell up to its chunk's end
constexpr unsigned long long kLookValue = (1ull << 62) - 1ull;

__device__ __forceinline__ unsigned long long load_acquire64(const unsigned long long* p) {
	unsigned long long v;
	asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}

// Wrap, binning, scan and (cell, id) sort of all molecules in one cooperative launch with three
// bounded grid barriers; returns at once unless a build was asked for this step. count[] and look[]
// are zero on entry and are left zero for the next launch (a launch that gave up on a wait leaves
// them to the host, which clears them with the timeout status).
//   1. wrap + cell + arrival rank: one atomic per cell and warp (the warp's molecules of a cell,
//      found by __match_any_sync, take consecutive ranks)
//   2. exclusive scan of the counts in one pass: CTA b sums the cells of its chunk, publishes the
//      sum, adds up its predecessors' published values back to the first complete prefix, 32 at a
//      time by one warp (decoupled look-back: every CTA of the cooperative grid is resident, so each
//      of these waits ends; each is bounded nonetheless) and publishes its own prefix
//   3. every molecule to its arrival slot in the other buffer, with its cell and previous slot;
//      counts and look-back words cleared for the next launch
//   4. one thread per slot: its rank by (id, previous slot) among its cell's slots, read from the
//      contiguous ids of the cell, and the molecule back into the current buffer at that rank (the
//      host's buffer roles stay fixed)
__global__ void __launch_bounds__(kRebuildThreads, 4) k_rebuild(RebuildArgs a) {
	__shared__ int s_flag;
	__shared__ int32_t s_excl;
	// (no flag: a build in every launch)
	if (threadIdx.x == 0)
		s_flag = ((!a.flag || *a.flag == a.step) && !(*((volatile int*) a.status) & kStatusTimeout)) ? 0 : 1;
	__syncthreads();
	if (s_flag) return;   // no build requested for this step
	if (blockIdx.x == 0 && threadIdx.x < 2 && a.brick_counts) a.brick_counts[threadIdx.x] = 0u;
	const int64_t nthreads = (int64_t) gridDim.x * blockDim.x;
	const int64_t tid = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	const int64_t nc = a.g.ncells;
	const int lane = threadIdx.x & 31;
	bool bad = false;
	// warp-uniform trip count (nthreads is a multiple of 32): every lane takes part in the match
	for (int64_t i0 = tid - lane; i0 < a.n; i0 += nthreads) {
		const int64_t i = i0 + lane;
		const bool valid = i < a.n;
		const int32_t c = valid ? bin_one(i, a.p.rx, a.p.ry, a.p.rz, a.g, bad) : -1;
		const unsigned peers = __match_any_sync(0xffffffffu, c);
		const int leader = __ffs(peers) - 1;
		int32_t base = 0;
		if (valid && lane == leader) base = atomicAdd(&a.count[c], __popc(peers));
		base = __shfl_sync(0xffffffffu, base, leader);
		if (valid) {
			a.cell[i] = c;
			a.rank[i] = base + __popc(peers & ((1u << lane) - 1u));
		}
	}
	if (bad) atomicOr(a.status, kStatusOutsideHalo);
	if (!grid_barrier(a.bar, a.status, a.timeout_ns, &s_flag)) return;
	// 2. one contiguous chunk of cells per CTA, scanned with the prefix of the chunks before it
	const int64_t per = (nc + gridDim.x - 1) / gridDim.x;
	const int64_t c0 = min((int64_t) blockIdx.x * per, nc), c1 = min(c0 + per, nc);
	{
		int32_t local = 0;
		for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) local += a.count[c];
		int32_t agg;
		// with at most one cell per thread this is already the chunk's own exclusive scan
		const int32_t lexcl = block_excl_scan(local, &agg);
		if (threadIdx.x < 32) {
			unsigned long long* look = a.look;
			const int b = (int) blockIdx.x;
			if (lane == 0) {
				__threadfence();
				atomicExch(look + b, (b == 0 ? kLookPrefix : kLookAggregate) | (unsigned long long) agg);
			}
			// predecessors b-1-lane, 32 per round; those before CTA 0 count as a zero prefix
			int64_t excl = 0;
			bool late = false;
			const uint64_t t0 = __shfl_sync(0xffffffffu, global_ns(), 0);
			for (int j = b - 1; j >= 0;) {
				const int idx = j - lane;
				const unsigned long long v = idx >= 0 ? load_acquire64(look + idx) : kLookPrefix;
				if (__any_sync(0xffffffffu, v == 0ull)) {
					// a predecessor of the window has not published yet
					late = __shfl_sync(0xffffffffu, (int64_t) (global_ns() - t0) > a.timeout_ns, 0);
					if (late) break;
					continue;
				}
				const unsigned pm = __ballot_sync(0xffffffffu, (v & kLookPrefix) != 0ull);
				const int first = pm ? __ffs(pm) - 1 : 32;   // the nearest complete prefix
				unsigned long long val = (lane <= first && idx >= 0) ? (v & kLookValue) : 0ull;
				for (int o = 16; o; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
				excl += (int64_t) val;
				if (pm) break;
				j -= 32;
			}
			if (lane == 0) {
				if (late) {
					atomicOr(a.status, kStatusTimeout);
					s_flag = 1;
				} else if (b > 0) {
					__threadfence();
					atomicExch(look + b, kLookPrefix | (unsigned long long) (excl + agg));
				}
				s_excl = (int32_t) excl;
				if (b == (int) gridDim.x - 1) a.start[nc] = (int32_t) (excl + agg);
			}
		}
		__syncthreads();
		if (s_flag) return;
		if (per <= (int64_t) blockDim.x) {
			if (c0 + threadIdx.x < c1) a.start[c0 + threadIdx.x] = s_excl + lexcl;
		} else {
			int32_t carry = s_excl;
			for (int64_t base = c0; base < c1; base += blockDim.x) {
				const int64_t c = base + threadIdx.x;
				const int32_t v = c < c1 ? a.count[c] : 0;
				int32_t tot;
				const int32_t excl = block_excl_scan(v, &tot);
				if (c < c1) a.start[c] = carry + excl;
				carry += tot;
			}
		}
	}
	if (!grid_barrier(a.bar, a.status, a.timeout_ns, &s_flag)) return;
	// 3. every molecule, all fields, to its arrival slot in the other buffer, with its cell and
	// previous slot; the counts and the look-back words are not read again in this launch. All loads
	// come before the stores (the compiler cannot tell the buffers apart).
	for (int64_t i = tid; i < a.n; i += nthreads) {
		const int32_t c = a.cell[i], rk = a.rank[i];
		const double x = a.p.rx[i], y = a.p.ry[i], z = a.p.rz[i];
		const double vx = a.p.vx[i], vy = a.p.vy[i], vz = a.p.vz[i];
		const uint64_t id = a.p.id[i];
		const int32_t ci = a.p.cid[i], ui = a.p.uidx[i];
		const int32_t s = a.start[c], e = a.start[c + 1];
		const int32_t slot = s + rk;
		a.q.rx[slot] = x;
		a.q.ry[slot] = y;
		a.q.rz[slot] = z;
		a.q.vx[slot] = vx;
		a.q.vy[slot] = vy;
		a.q.vz[slot] = vz;
		a.q.id[slot] = id;
		a.q.cid[slot] = ci;
		a.q.uidx[slot] = ui;
		a.slot[slot] = make_int4(c, s, e, (int32_t) i);
		for (int k = 0; k < a.nx; k++) a.xt[(int64_t) k * a.n + slot] = a.xs[(int64_t) k * a.n + i];
	}
	for (int64_t c = tid; c < nc; c += nthreads) a.count[c] = 0;
	if (threadIdx.x == 0) a.look[blockIdx.x] = 0ull;
	if (!grid_barrier(a.bar, a.status, a.timeout_ns, &s_flag)) return;
	// 4. slot t's place in its cell, the cell's slots with a smaller (id, previous slot), read from
	// the cell's contiguous ids; the molecule back into the current buffer there
	for (int64_t t = tid; t < a.n; t += nthreads) {
		const int4 sl = a.slot[t];
		const double x = a.q.rx[t], y = a.q.ry[t], z = a.q.rz[t];
		const double vx = a.q.vx[t], vy = a.q.vy[t], vz = a.q.vz[t];
		const uint64_t key = a.q.id[t];
		const int32_t ci = a.q.cid[t], ui = a.q.uidx[t];
		int32_t pos = 0;
#pragma unroll 4
		for (int32_t k = sl.y; k < sl.z; k++) {
			const uint64_t ok = a.q.id[k];
			// equal ids (not in valid input) keep the order of their previous slots
			pos += ok < key ? 1 : ((ok == key && a.slot[k].w < sl.w) ? 1 : 0);
		}
		const int32_t to = sl.y + pos;
		a.p.rx[to] = x;
		a.p.ry[to] = y;
		a.p.rz[to] = z;
		a.p.vx[to] = vx;
		a.p.vy[to] = vy;
		a.p.vz[to] = vz;
		a.p.id[to] = key;
		a.p.cid[to] = ci;
		a.p.uidx[to] = ui;
		a.cell[to] = sl.x;
		a.perm[to] = sl.w;   // the slot's molecule before the rebuild, for state kept beside p
		for (int k = 0; k < a.nx; k++) a.xs[(int64_t) k * a.n + to] = a.xt[(int64_t) k * a.n + t];
	}
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned) ((n + t - 1) / t); }

}  // namespace

cudaError_t launch_bin(Context* c, bool permute_forces) {
	const int64_t n = c->n, nc = c->g.ncells;
	cudaStream_t s = c->stream;
	prof_begin(c, 0);
	cudaMemsetAsync(c->cell_count, 0, sizeof(int32_t) * nc, s);
	if (n > 0) k_bin_cells<<<blocks_for(n, 256), 256, 0, s>>>(n, c->p.rx, c->p.ry, c->p.rz, c->g, c->cell, c->rank,
	                                                          c->cell_count, c->status);
	int64_t nb = (nc + kScanBlock - 1) / kScanBlock;
	k_scan_local<<<(unsigned) nb, 256, 0, s>>>(nc, c->cell_count, c->cell_start, c->scan_tmp);
	k_scan_sums<<<1, 1024, 0, s>>>(nb, c->scan_tmp);
	k_scan_add<<<blocks_for(nc, 256), 256, 0, s>>>(nc, c->cell_start, c->scan_tmp, nb);
	int launches = 4;
	if (n > 0) {
		k_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, c->cell, c->rank, c->cell_start, c->perm);
		k_cell_sort<<<blocks_for(nc * 32, 256), 256, 0, s>>>(nc, c->cell_start, c->perm, c->p, c->q, c->rank,
		                                                     permute_forces);
		launches += 2;
	}
	cudaError_t e = cudaGetLastError();
	// the sorted cell of each particle was written into `rank`; swap buffers
	Particles t = c->p;
	c->p = c->q;
	c->q = t;
	int32_t* tc = c->cell;
	c->cell = c->rank;
	c->rank = tc;
	prof_end(c, 0, launches);
	return e;
}

cudaError_t launch_rebuild(Context* c, const Grid& g, double* extra, double* scratch, int nextra, bool always) {
	// co-resident CTAs per SM of k_rebuild, per device (the occupancy query is a host call of
	// several microseconds, paid once per device)
	static std::mutex mu;
	static int per_sm_of[kMaxDevices] = {};
	int per_sm = 0;
	{
		std::lock_guard<std::mutex> lock(mu);
		if (c->device >= 0 && c->device < kMaxDevices) per_sm = per_sm_of[c->device];
	}
	if (per_sm == 0) {
		cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rebuild, kRebuildThreads, 0);
		if (e != cudaSuccess) return e;
		if (per_sm < 1) per_sm = 1;
		std::lock_guard<std::mutex> lock(mu);
		if (c->device >= 0 && c->device < kMaxDevices) per_sm_of[c->device] = per_sm;
	}
	const int max_ctas = per_sm * c->num_sms;
	prof_begin(c, 0);
	RebuildArgs a{};
	a.n = c->n;
	a.g = g;
	a.p = c->p;
	a.q = c->q;
	a.cell = c->cell;
	a.rank = c->rank;
	a.perm = c->perm;
	a.slot = c->rb_slot;
	a.count = c->rb_count;
	a.start = c->cell_start;
	a.look = c->rb_look;
	a.status = c->status;
	a.flag = always ? nullptr : c->rebuild;
	a.step = c->step_id;
	a.bar = c->bar;
	a.timeout_ns = 2000000000LL;
	a.brick_counts = c->brick_counts;
	a.xs = extra;
	a.xt = scratch;
	a.nx = extra ? nextra : 0;
	// one chunk sum per CTA; no more CTAs than the molecules and cells need (a co-resident grid of
	// the whole device would keep every other stream's kernels waiting, also in steps it is gated off)
	const int64_t work = std::max<int64_t>(c->n, g.ncells);
	int grid = (int) std::min<int64_t>(max_ctas, (work + kRebuildThreads - 1) / kRebuildThreads);
	if (grid > c->rb_look_cap) grid = c->rb_look_cap;
	if (grid < 1) grid = 1;
	cudaLaunchConfig_t cfg{};
	cfg.gridDim = dim3((unsigned) grid);
	cfg.blockDim = dim3(kRebuildThreads);
	cfg.stream = c->stream;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeCooperative;
	attr[0].val.cooperative = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	cudaError_t e = cudaLaunchKernelEx(&cfg, k_rebuild, a);
	prof_end(c, 0, 1);
	return e;
}

}  // namespace mdgpu
