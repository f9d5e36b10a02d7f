// Single-box pair kernel: one CTA per brick of 2x2x2 linked cells (the per-brick work is
// brick::pairs in brick.cuh, which also documents the staging, filter and compute passes).
#include <cuda_runtime.h>

#include "brick.cuh"
#include "md_internal.h"

namespace mdgpu {
namespace {

constexpr int kListCap = 64;

template <bool kFP64, bool kSingle, bool kLjIsRc>
__global__ void __launch_bounds__(brick::kThreads, 2)
    k_pairs_brick(brick::Const p, brick::Box bx, const double* __restrict__ rx, const double* __restrict__ ry,
                  const double* __restrict__ rz, const int32_t* __restrict__ cid,
                  const int32_t* __restrict__ cstart, const PairParams* __restrict__ pp,
                  double* __restrict__ fx, double* __restrict__ fy, double* __restrict__ fz,
                  double* __restrict__ partials, int* __restrict__ status) {
	extern __shared__ __align__(16) unsigned char smem[];
	brick::load_params(smem, brick::layout(p.s_cap, kFP64, kListCap), pp, p.ns);
	__syncthreads();
	brick::pairs<kFP64, kSingle, kLjIsRc, kListCap>(p, bx, blockIdx.x, blockIdx.x, smem, rx, ry, rz, cid, cstart, fx,
	                                                fy, fz, partials, status);
}

}  // namespace

cudaError_t launch_pairs_brick(Context* c) {
	const bool fp64 = c->precision == MDGPU_FP64;
	brick::Box bx{};
	brick::init_box(bx, c->g, c->rc, 0);
	// shared-memory capacity: two CTAs per SM
	static int max_optin = -1;
	if (max_optin < 0) cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
	size_t budget = 110 * 1024;
	if (budget > (size_t) max_optin) budget = (size_t) max_optin;
	const int s_cap = brick::capacity_for(budget, fp64, kListCap);
	const brick::Const p = brick::make_const(c->sp.n, s_cap, c->rc, c->rc_lj);
	const size_t bytes = brick::layout(s_cap, fp64, kListCap).total;
	const int nbricks = bx.nb[0] * bx.nb[1] * bx.nb[2];
	prof_begin(c, 1);
	cudaError_t e;
	const bool single = c->sp.n == 1;
	auto go = [&](auto kern) {
		cudaError_t r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bytes);
		if (r == cudaSuccess)
			kern<<<nbricks, brick::kThreads, bytes, c->stream>>>(p, bx, c->p.rx, c->p.ry, c->p.rz, c->p.cid,
			                                                     c->cell_start, c->d_pp, c->p.fx, c->p.fy, c->p.fz,
			                                                     c->partials, c->status);
		return r;
	};
	const bool ljrc = c->rc_lj == c->rc;
	if (fp64)
		e = single ? go(k_pairs_brick<true, true, false>) : go(k_pairs_brick<true, false, false>);
	else if (ljrc)
		e = single ? go(k_pairs_brick<false, true, true>) : go(k_pairs_brick<false, false, true>);
	else
		e = single ? go(k_pairs_brick<false, true, false>) : go(k_pairs_brick<false, false, false>);
	if (e == cudaSuccess) e = cudaGetLastError();
	prof_end(c, 1, 1);
	if (e != cudaSuccess) return e;
	return launch_reduce(c, nbricks, c->scalars, 3);
}

}  // namespace mdgpu
