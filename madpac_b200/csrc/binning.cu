// Linked-cell binning by counting sort into a cell-ordered structure of arrays.
//
// Per update (LinkedCells::update, particleContainer/LinkedCells.cpp:165-180, paths relative to
// madpac/mardyn/):
//   1. bin_cells:  periodic wrap of each coordinate (r<0 -> r+L, r>=L -> r-L: the position of the
//                  halo image that survives DomainDecompDummy::exchangeMolecules +
//                  LinkedCells::deleteOuterParticles, parallel/DomainDecompDummy.cpp:64-70, 93-99,
//                  LinkedCells.cpp:356-369), the cell coordinate floor((r - haloMin)/cellLength)
//                  in IEEE double with no contraction (LinkedCells.cpp:543), and an atomic
//                  arrival rank per cell.
//   2. scan:       exclusive prefix sum of the cell counts (two-level).
//   3. scatter:    slot = cell_start + rank (arrival order, not deterministic).
//   4. cell_sort:  one warp per cell orders its molecules by id and gathers every field into
//                  the other buffer, so the final order (cell, id) does not depend on timing.
#include <cuda_runtime.h>

#include "md_internal.h"

namespace mdgpu {
namespace {

constexpr int kScanBlock = 1024;   // elements per scan block (256 threads x 4)

__global__ void k_bin_cells(int64_t n, double* __restrict__ rx, double* __restrict__ ry,
                            double* __restrict__ rz, Grid g, int32_t* __restrict__ cell,
                            int32_t* __restrict__ rank, int32_t* __restrict__ count, int* status, const int* gate) {
	if (gate && *gate == 0) return;
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	double r[3] = {rx[i], ry[i], rz[i]};
	int ci[3];
	bool bad = false;
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
	if (bad) atomicOr(status, kStatusOutsideHalo);
	if (r[0] != rx[i]) rx[i] = r[0];
	if (r[1] != ry[i]) ry[i] = r[1];
	if (r[2] != rz[i]) rz[i] = r[2];
	int32_t c = (int32_t) (((int64_t) ci[2] * g.nc[1] + ci[1]) * g.nc[0] + ci[0]);
	cell[i] = c;
	rank[i] = atomicAdd(&count[c], 1);
}

// Block-local exclusive scan of kScanBlock counts; block totals go to sums.
__global__ void k_scan_local(int64_t n, const int32_t* __restrict__ in, int32_t* __restrict__ out,
                             int32_t* __restrict__ sums, const int* gate) {
	if (gate && *gate == 0) return;
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

// Single block: exclusive scan of the block totals, total appended at sums[nb].
__global__ void k_scan_sums(int64_t nb, int32_t* sums, const int* gate) {
	if (gate && *gate == 0) return;
	__shared__ int32_t carry;
	if (threadIdx.x == 0) carry = 0;
	__syncthreads();
	for (int64_t base = 0; base < nb; base += blockDim.x) {
		int64_t i = base + threadIdx.x;
		int32_t v = i < nb ? sums[i] : 0;
		int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
		__shared__ int32_t wt[32];
		int32_t inc = v;
		for (int o = 1; o < 32; o <<= 1) {
			int32_t y = __shfl_up_sync(0xffffffffu, inc, o);
			if (lane >= o) inc += y;
		}
		if (lane == 31) wt[warp] = inc;
		__syncthreads();
		if (warp == 0) {
			int nw = blockDim.x >> 5;
			int32_t w = lane < nw ? wt[lane] : 0;
			for (int o = 1; o < 32; o <<= 1) {
				int32_t y = __shfl_up_sync(0xffffffffu, w, o);
				if (lane >= o) w += y;
			}
			wt[lane] = w;
		}
		__syncthreads();
		int32_t excl = carry + inc - v + (warp > 0 ? wt[warp - 1] : 0);
		if (i < nb) sums[i] = excl;
		__syncthreads();
		if (threadIdx.x == blockDim.x - 1) carry = excl + v;
		__syncthreads();
	}
	if (threadIdx.x == 0) sums[nb] = carry;
}

__global__ void k_scan_add(int64_t n, int32_t* __restrict__ out, const int32_t* __restrict__ sums, int64_t nb,
                           const int* gate) {
	if (gate && *gate == 0) return;
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] += sums[i / kScanBlock];
	if (i == 0) out[n] = sums[nb];
}

__global__ void k_scatter(int64_t n, const int32_t* __restrict__ cell, const int32_t* __restrict__ rank,
                          const int32_t* __restrict__ start, int32_t* __restrict__ perm, const int* gate) {
	if (gate && *gate == 0) return;
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) perm[start[cell[i]] + rank[i]] = (int32_t) i;
}

__device__ __forceinline__ bool key_less(uint64_t ka, int32_t sa, uint64_t kb, int32_t sb) {
	return ka < kb || (ka == kb && sa < sb);
}

// One warp per cell: order the cell's molecules by (id, previous slot) and gather all fields.
__global__ void k_cell_sort(int64_t ncells, const int32_t* __restrict__ start, const int32_t* __restrict__ perm,
                            Particles src, Particles dst, int32_t* __restrict__ cell_out, bool with_forces,
                            const int* gate) {
	if (gate && *gate == 0) return;
	int64_t c = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	int lane = threadIdx.x & 31;
	if (c >= ncells) return;
	int32_t s = start[c], m = start[c + 1] - s;
	for (int32_t e0 = 0; e0 < m; e0 += 32) {
		int32_t e = e0 + lane;
		int32_t from = -1;
		uint64_t key = 0;
		int32_t pos = 0;
		if (e < m) {
			from = perm[s + e];
			key = src.id[from];
		}
		if (m <= 32) {
			for (int k = 0; k < m; k++) {
				uint64_t ok = __shfl_sync(0xffffffffu, key, k);
				int32_t of = __shfl_sync(0xffffffffu, from, k);
				if (key_less(ok, of, key, from)) pos++;
			}
		} else if (e < m) {
			for (int32_t k = 0; k < m; k++) {
				int32_t of = perm[s + k];
				if (key_less(src.id[of], of, key, from)) pos++;
			}
		}
		if (e < m) {
			int32_t to = s + pos;
			dst.rx[to] = src.rx[from];
			dst.ry[to] = src.ry[from];
			dst.rz[to] = src.rz[from];
			dst.vx[to] = src.vx[from];
			dst.vy[to] = src.vy[from];
			dst.vz[to] = src.vz[from];
			if (with_forces) {
				dst.fx[to] = src.fx[from];
				dst.fy[to] = src.fy[from];
				dst.fz[to] = src.fz[from];
			}
			dst.id[to] = key;
			dst.cid[to] = src.cid[from];
			dst.uidx[to] = src.uidx[from];
			cell_out[to] = (int32_t) c;
		}
	}
}

// Gated mode: the sorted arrays (and their cells) back into the current buffer.
__global__ void k_copy_back(int64_t n, Particles src, Particles dst, const int32_t* __restrict__ cell_src,
                            int32_t* __restrict__ cell_dst, const int* gate) {
	if (*gate == 0) return;
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	dst.rx[i] = src.rx[i];
	dst.ry[i] = src.ry[i];
	dst.rz[i] = src.rz[i];
	dst.vx[i] = src.vx[i];
	dst.vy[i] = src.vy[i];
	dst.vz[i] = src.vz[i];
	dst.id[i] = src.id[i];
	dst.cid[i] = src.cid[i];
	dst.uidx[i] = src.uidx[i];
	cell_dst[i] = cell_src[i];
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned) ((n + t - 1) / t); }

}  // namespace

cudaError_t launch_bin(Context* c, bool permute_forces, const int* gate, const Grid* grid) {
	const Grid& g = grid ? *grid : c->g;
	const int64_t n = c->n, nc = g.ncells;
	cudaStream_t s = c->stream;
	prof_begin(c, 0);
	cudaMemsetAsync(c->cell_count, 0, sizeof(int32_t) * nc, s);
	if (n > 0) k_bin_cells<<<blocks_for(n, 256), 256, 0, s>>>(n, c->p.rx, c->p.ry, c->p.rz, g, c->cell, c->rank,
	                                                          c->cell_count, c->status, gate);
	int64_t nb = (nc + kScanBlock - 1) / kScanBlock;
	k_scan_local<<<(unsigned) nb, 256, 0, s>>>(nc, c->cell_count, c->cell_start, c->scan_tmp, gate);
	k_scan_sums<<<1, 1024, 0, s>>>(nb, c->scan_tmp, gate);
	k_scan_add<<<blocks_for(nc, 256), 256, 0, s>>>(nc, c->cell_start, c->scan_tmp, nb, gate);
	int launches = 4;
	if (n > 0) {
		k_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, c->cell, c->rank, c->cell_start, c->perm, gate);
		k_cell_sort<<<blocks_for(nc * 32, 256), 256, 0, s>>>(nc, c->cell_start, c->perm, c->p, c->q, c->rank,
		                                                     permute_forces, gate);
		launches += 2;
		if (gate) {
			k_copy_back<<<blocks_for(n, 256), 256, 0, s>>>(n, c->q, c->p, c->rank, c->cell, gate);
			launches += 1;
		}
	}
	cudaError_t e = cudaGetLastError();
	if (!gate) {
		// the sorted cell of each particle was written into `rank`; swap buffers
		Particles t = c->p;
		c->p = c->q;
		c->q = t;
		int32_t* tc = c->cell;
		c->cell = c->rank;
		c->rank = tc;
	}
	prof_end(c, 0, launches);
	return e;
}

}  // namespace mdgpu
