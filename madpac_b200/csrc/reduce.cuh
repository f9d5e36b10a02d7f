// Fixed-order (deterministic) warp and block reductions shared by the kernels.
#pragma once

#include "md_internal.h"

namespace mdgpu {

__device__ __forceinline__ double warp_sum(double v) {
	for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
	return v;
}

// Block-wide sum of three doubles into partials[slot*4 + k] (blockDim.x <= kReduceBlock).
__device__ __forceinline__ void block_sum3_at(double a, double b, double c, double* partials, int64_t slot) {
	__shared__ double sh[3][kReduceBlock / 32];
	a = warp_sum(a);
	b = warp_sum(b);
	c = warp_sum(c);
	int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (lane == 0) {
		sh[0][warp] = a;
		sh[1][warp] = b;
		sh[2][warp] = c;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		double s0 = 0, s1 = 0, s2 = 0;
		for (int w = 0; w < (int) (blockDim.x >> 5); w++) {
			s0 += sh[0][w];
			s1 += sh[1][w];
			s2 += sh[2][w];
		}
		partials[slot * 4 + 0] = s0;
		partials[slot * 4 + 1] = s1;
		partials[slot * 4 + 2] = s2;
		partials[slot * 4 + 3] = 0.0;
	}
}

__device__ __forceinline__ void block_sum3(double a, double b, double c, double* partials) {
	block_sum3_at(a, b, c, partials, blockIdx.x);
}

}  // namespace mdgpu
