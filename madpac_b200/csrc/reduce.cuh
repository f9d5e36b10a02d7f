// Fixed-order (deterministic) warp and block reductions shared by the kernels.
#pragma once

#include "md_internal.h"

namespace mdgpu {

__device__ __forceinline__ double warp_sum(double v) {
	for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
	return v;
}

// Block-wide sums of three (or four) doubles into partials[slot*4 + k] (blockDim.x <= kReduceBlock).
__device__ __forceinline__ void block_sum3_at(double a, double b, double c, double* partials, int64_t slot,
                                              double d = 0.0) {
	__shared__ double sh[4][kReduceBlock / 32];
	a = warp_sum(a);
	b = warp_sum(b);
	c = warp_sum(c);
	d = warp_sum(d);
	int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (lane == 0) {
		sh[0][warp] = a;
		sh[1][warp] = b;
		sh[2][warp] = c;
		sh[3][warp] = d;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
		for (int w = 0; w < (int) (blockDim.x >> 5); w++) {
			s0 += sh[0][w];
			s1 += sh[1][w];
			s2 += sh[2][w];
			s3 += sh[3][w];
		}
		partials[slot * 4 + 0] = s0;
		partials[slot * 4 + 1] = s1;
		partials[slot * 4 + 2] = s2;
		partials[slot * 4 + 3] = s3;
	}
}

__device__ __forceinline__ void block_sum3(double a, double b, double c, double* partials) {
	block_sum3_at(a, b, c, partials, blockIdx.x);
}

// Run by every thread of every block after the block's partials (written by its thread 0) are in
// place: the last block to arrive (ticket counter, reset here) sums the nparts partials in a fixed
// order into out[0..nval) -- the same sums run to run, without a separate reduction launch.
// Returns true in the block that did the sum (blockDim.x <= kReduceBlock).
__device__ __forceinline__ bool last_block_sum(unsigned* counter, const double* partials, int64_t nparts, int nval,
                                               double* out) {
	__shared__ int s_last;
	__shared__ double sh[4][kReduceBlock / 32];
	__threadfence();
	__syncthreads();
	if (threadIdx.x == 0) s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
	__syncthreads();
	if (!s_last) return false;
	__threadfence();
	double acc[4] = {0, 0, 0, 0};
	for (int64_t b = threadIdx.x; b < nparts; b += blockDim.x)
		for (int k = 0; k < nval; k++) acc[k] += __ldcg(partials + b * 4 + k);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int k = 0; k < nval; k++) {
		const double v = warp_sum(acc[k]);
		if (lane == 0) sh[k][warp] = v;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int k = 0; k < nval; k++) {
			double t = 0;
			for (int w = 0; w < (int) (blockDim.x >> 5); w++) t += sh[k][w];
			out[k] = t;
		}
		*counter = 0u;
	}
	return true;
}

}  // namespace mdgpu
