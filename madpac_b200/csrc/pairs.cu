// Lennard-Jones 12-6 pair forces, potential energy and virial over the linked cells: the simple
// gather kernel (one thread per molecule, operands straight from global memory) and the final
// fixed-order reduction. The default pair kernel is the shared-memory brick kernel of
// pairs_brick.cu; this one is kept as an independent second implementation for the tests.
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
#include "pair_common.cuh"
#include "reduce.cuh"

namespace mdgpu {
namespace {


template <bool kMixed>
__global__ void __launch_bounds__(kReduceBlock) k_pairs_gather(int64_t n, const double* __restrict__ rx,
                                                               const double* __restrict__ ry,
                                                               const double* __restrict__ rz,
                                                               const int32_t* __restrict__ cid,
                                                               const int32_t* __restrict__ start, Grid g,
                                                               const PairParams* __restrict__ pp,
                                                               double* __restrict__ fx, double* __restrict__ fy,
                                                               double* __restrict__ fz, double* partials,
                                                               int* status) {
	constexpr int KK = kMaxSpecies * kMaxSpecies;
	__shared__ double s_par[3 * KK];
	const int ns = pp->ns;
	for (int k = threadIdx.x; k < ns * ns; k += blockDim.x) {
		s_par[k] = pp->eps24[k];
		s_par[KK + k] = pp->sig2[k];
		s_par[2 * KK + k] = pp->shift6[k];
	}
	__syncthreads();
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	double U = 0.0, W = 0.0, np = 0.0;
	bool same = false;
	if (i < n) {
		const PairSums s = gather_pairs<kMixed>(i, rx, ry, rz, cid, start, g, s_par, ns, pp->rc2, pp->rclj2);
		fx[i] = s.F[0];
		fy[i] = s.F[1];
		fz[i] = s.F[2];
		U = s.U;
		W = s.W;
		np = s.np;
		same = s.same;
		if (!(s.F[0] == s.F[0] && s.F[1] == s.F[1] && s.F[2] == s.F[2]) || isinf(s.F[0]) || isinf(s.F[1]) ||
		    isinf(s.F[2]))
			atomicOr(status, kStatusNonFinite);
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

cudaError_t launch_pairs_brick(Context* c);

cudaError_t launch_pairs(Context* c) {
	if (c->pair_kernel == 0 && c->n < (int64_t(1) << 28)) return launch_pairs_brick(c);
	prof_begin(c, 1);
	int64_t nb = (c->n + kReduceBlock - 1) / kReduceBlock;
	if (nb == 0) nb = 1;
	if (c->precision == MDGPU_MIXED)
		k_pairs_gather<true><<<(unsigned) nb, kReduceBlock, 0, c->stream>>>(
		    c->n, c->p.rx, c->p.ry, c->p.rz, c->p.cid, c->cell_start, c->g, c->d_pp, c->p.fx, c->p.fy, c->p.fz,
		    c->partials, c->status);
	else
		k_pairs_gather<false><<<(unsigned) nb, kReduceBlock, 0, c->stream>>>(
		    c->n, c->p.rx, c->p.ry, c->p.rz, c->p.cid, c->cell_start, c->g, c->d_pp, c->p.fx, c->p.fy, c->p.fz,
		    c->partials, c->status);
	cudaError_t e = cudaGetLastError();
	prof_end(c, 1, 1);
	if (e != cudaSuccess) return e;
	return launch_reduce(c, nb, c->scalars, 3);
}

}  // namespace mdgpu
