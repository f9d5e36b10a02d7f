// Lennard-Jones 12-6 pair forces, potential energy and virial over the linked cells.
//
// Every molecule i gathers from all molecules j of the 27 cells around its own (periodic images
// are the neighbour cell's molecules shifted by +-L, computed as the reference computes a halo
// image's position: r_j + L or r_j - L, parallel/DomainDecompDummy.cpp:64-70, 93-99). Each
// unordered pair is therefore evaluated from both sides; the energy and virial are halved at the
// end, which reproduces the reference's "count every pair once" rule (BlockTraverse.cpp:279-285,
// 310; ParticlePairs2PotForceAdapter.h:91-103).
//
// The per-pair arithmetic follows PotForceLJ (molecules/potforce.h:41-53) and the LJ block of
// PotForce (potforce.h:328-363): drm = r_i - r_j, dd = drm.drm, invdr2 = 1/dd,
// lj6 = (sig2*invdr2)^3, lj12 = lj6^2, u6 = eps24*(lj12-lj6) + shift6,
// f = eps24*(lj12 + (lj12-lj6))*invdr2 * drm, virial += drm.f, with the cutoff tests dd < rc^2
// (pair) and dd < rcLJ^2 (LJ), both strict (BlockTraverse.cpp:155).
// MDGPU_FP64 evaluates it in double with the reference's operation order and no contraction;
// MDGPU_MIXED rounds drm to float and evaluates the LJ terms in float, accumulating in double.
#include <cuda_runtime.h>

#include "md_internal.h"
#include "reduce.cuh"

namespace mdgpu {
namespace {


template <bool kMixed>
__global__ void __launch_bounds__(kReduceBlock) k_pairs_gather(int64_t n, const double* __restrict__ rx,
                                                               const double* __restrict__ ry,
                                                               const double* __restrict__ rz,
                                                               const int32_t* __restrict__ cid,
                                                               const int32_t* __restrict__ cell,
                                                               const int32_t* __restrict__ start, Grid g,
                                                               const PairParams* __restrict__ pp,
                                                               double* __restrict__ fx, double* __restrict__ fy,
                                                               double* __restrict__ fz, double* partials,
                                                               int* status) {
	__shared__ double s_eps24[kMaxSpecies * kMaxSpecies], s_sig2[kMaxSpecies * kMaxSpecies],
	    s_shift6[kMaxSpecies * kMaxSpecies];
	int ns = pp->ns;
	for (int k = threadIdx.x; k < ns * ns; k += blockDim.x) {
		s_eps24[k] = pp->eps24[k];
		s_sig2[k] = pp->sig2[k];
		s_shift6[k] = pp->shift6[k];
	}
	__syncthreads();
	const double rc2 = pp->rc2, rclj2 = pp->rclj2;
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	double U = 0.0, W = 0.0, np = 0.0;
	bool same = false;
	if (i < n) {
		const double xi = rx[i], yi = ry[i], zi = rz[i];
		const int ti = cid[i];
		const int c = cell[i];
		const int cx = c % g.nc[0], cy = (c / g.nc[0]) % g.nc[1], cz = c / (g.nc[0] * g.nc[1]);
		double Fx = 0.0, Fy = 0.0, Fz = 0.0;
		for (int dz = -1; dz <= 1; dz++) {
			int z = cz + dz;
			double sz = 0.0;
			if (z < 0) { z += g.nc[2]; sz = -g.L[2]; }
			else if (z >= g.nc[2]) { z -= g.nc[2]; sz = g.L[2]; }
			for (int dy = -1; dy <= 1; dy++) {
				int y = cy + dy;
				double sy = 0.0;
				if (y < 0) { y += g.nc[1]; sy = -g.L[1]; }
				else if (y >= g.nc[1]) { y -= g.nc[1]; sy = g.L[1]; }
				for (int dx = -1; dx <= 1; dx++) {
					int x = cx + dx;
					double sx = 0.0;
					if (x < 0) { x += g.nc[0]; sx = -g.L[0]; }
					else if (x >= g.nc[0]) { x -= g.nc[0]; sx = g.L[0]; }
					const int nb = (z * g.nc[1] + y) * g.nc[0] + x;
					const bool shifted = (sx != 0.0) || (sy != 0.0) || (sz != 0.0);
					const int j0 = start[nb], j1 = start[nb + 1];
					for (int j = j0; j < j1; j++) {
						if (j == i && !shifted) continue;
						double xj = rx[j], yj = ry[j], zj = rz[j];
						if (shifted) {
							xj = __dadd_rn(xj, sx);
							yj = __dadd_rn(yj, sy);
							zj = __dadd_rn(zj, sz);
						}
						const double d0 = __dsub_rn(xi, xj), d1 = __dsub_rn(yi, yj), d2 = __dsub_rn(zi, zj);
						const double dd = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
						if (!(dd < rc2)) continue;
						np += 1.0;
						if (dd == 0.0) same = true;
						if (!(dd < rclj2)) continue;
						const int pk = ti * ns + cid[j];
						if (!kMixed) {
							const double eps24 = s_eps24[pk], sig2 = s_sig2[pk];
							const double invdr2 = __ddiv_rn(1.0, dd);
							double lj6 = __dmul_rn(sig2, invdr2);
							lj6 = __dmul_rn(__dmul_rn(lj6, lj6), lj6);
							const double lj12 = __dmul_rn(lj6, lj6);
							const double lj12m6 = __dsub_rn(lj12, lj6);
							const double u = __dadd_rn(__dmul_rn(eps24, lj12m6), s_shift6[pk]);
							const double fac = __dmul_rn(__dmul_rn(eps24, __dadd_rn(lj12, lj12m6)), invdr2);
							const double f0 = __dmul_rn(fac, d0), f1 = __dmul_rn(fac, d1), f2 = __dmul_rn(fac, d2);
							Fx += f0;
							Fy += f1;
							Fz += f2;
							U += u;
							W = __dadd_rn(W, __dadd_rn(__dadd_rn(__dmul_rn(d0, f0), __dmul_rn(d1, f1)), __dmul_rn(d2, f2)));
						} else {
							const float e0 = (float) d0, e1 = (float) d1, e2 = (float) d2;
							const float ddf = e0 * e0 + e1 * e1 + e2 * e2;
							const float eps24 = (float) s_eps24[pk], sig2 = (float) s_sig2[pk];
							const float invdr2 = 1.0f / ddf;
							float lj6 = sig2 * invdr2;
							lj6 = lj6 * lj6 * lj6;
							const float lj12 = lj6 * lj6;
							const float lj12m6 = lj12 - lj6;
							const float u = eps24 * lj12m6;
							const float fac = eps24 * (lj12 + lj12m6) * invdr2;
							const float f0 = fac * e0, f1 = fac * e1, f2 = fac * e2;
							Fx += (double) f0;
							Fy += (double) f1;
							Fz += (double) f2;
							U += (double) u + s_shift6[pk];
							W += (double) (e0 * f0 + e1 * f1 + e2 * f2);
						}
					}
				}
			}
		}
		fx[i] = Fx;
		fy[i] = Fy;
		fz[i] = Fz;
		if (!(Fx == Fx && Fy == Fy && Fz == Fz) || isinf(Fx) || isinf(Fy) || isinf(Fz)) atomicOr(status, kStatusNonFinite);
	}
	if (same) atomicOr(status, kStatusSamePosition);
	block_sum3(U, W, np, partials);
}

// One block sums the per-block partials in a fixed order into out[0..2].
__global__ void k_reduce_partials(int64_t nblocks, const double* __restrict__ partials, double* out, int nval) {
	__shared__ double sh[4][1024 / 32];
	double acc[4] = {0, 0, 0, 0};
	for (int64_t b = threadIdx.x; b < nblocks; b += blockDim.x)
		for (int k = 0; k < nval; k++) acc[k] += partials[b * 4 + k];
	int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int k = 0; k < nval; k++) {
		double v = warp_sum(acc[k]);
		if (lane == 0) sh[k][warp] = v;
	}
	__syncthreads();
	if (threadIdx.x == 0)
		for (int k = 0; k < nval; k++) {
			double s = 0;
			for (int w = 0; w < (int) (blockDim.x >> 5); w++) s += sh[k][w];
			out[k] = s;
		}
}

}  // namespace

// Exposed for the integration kernels, which reuse the fixed-order reduction.
cudaError_t launch_reduce(Context* c, int64_t nblocks, double* out, int nval) {
	k_reduce_partials<<<1, 1024, 0, c->stream>>>(nblocks, c->partials, out, nval);
	count_launches(c, 1);
	return cudaGetLastError();
}

cudaError_t launch_pairs(Context* c) {
	prof_begin(c, 1);
	int64_t nb = (c->n + kReduceBlock - 1) / kReduceBlock;
	if (nb == 0) nb = 1;
	if (c->precision == MDGPU_MIXED)
		k_pairs_gather<true><<<(unsigned) nb, kReduceBlock, 0, c->stream>>>(
		    c->n, c->p.rx, c->p.ry, c->p.rz, c->p.cid, c->cell, c->cell_start, c->g, c->d_pp, c->p.fx, c->p.fy,
		    c->p.fz, c->partials, c->status);
	else
		k_pairs_gather<false><<<(unsigned) nb, kReduceBlock, 0, c->stream>>>(
		    c->n, c->p.rx, c->p.ry, c->p.rz, c->p.cid, c->cell, c->cell_start, c->g, c->d_pp, c->p.fx, c->p.fy,
		    c->p.fz, c->partials, c->status);
	cudaError_t e = cudaGetLastError();
	prof_end(c, 1, 1);
	if (e != cudaSuccess) return e;
	return launch_reduce(c, nb, c->scalars, 3);
}

}  // namespace mdgpu
