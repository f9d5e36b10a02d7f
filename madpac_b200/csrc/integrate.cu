// Leapfrog (velocity Verlet) update, velocity scaling and the per-step record of mdgpu_run.
//
// The translational updates follow Molecule::upd_preF (molecules/Molecule.cpp:128-135) and
// Molecule::upd_postF (Molecule.cpp:193-205) operation by operation, with explicit
// round-to-nearest intrinsics so that no multiply-add contraction changes a bit:
//   pre:  v = vcorr*v + dtInv2m*F;  r += dt*v           (dtInv2m = (0.5*dt)/m)
//   post: v += dtInv2m*F;  sum m*(v0^2+v1^2+v2^2)       (dtInv2m = dt_half/m)
// For single-site LJ molecules the quaternion and angular-momentum parts of those functions
// leave r and v untouched (no torque, zero inertia), so they are not evaluated.
#include <cuda_runtime.h>

#include <algorithm>

#include "md_internal.h"
#include "reduce.cuh"

namespace mdgpu {
namespace {

struct SpeciesScale {
	double dtInv2m[kMaxSpecies];
	double mass[kMaxSpecies];
};

// Verlet-skin check of the pre-kick: the positions at the last build, the squared half skin, and
// the step id written to *flag when a molecule moved farther.
// With pruned lists, dmax receives the largest squared drift (float bits, rounded up).
struct SkinCheck {
	const double *rx, *ry, *rz;
	double half2;
	int* flag;
	int id;
	unsigned* dmax;
};

__global__ void __launch_bounds__(kReduceBlock) k_leapfrog_pre(int64_t n, Particles p, SpeciesScale s, double dt,
                                                              double vcorr, SkinCheck sk) {
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	const bool in = i < n;
	unsigned dm = 0u;
	if (in) {
		// every load first: the arrays may alias as far as the compiler knows
		const double a = s.dtInv2m[p.cid[i]];
		const double vx0 = p.vx[i], vy0 = p.vy[i], vz0 = p.vz[i];
		const double fx = p.fx[i], fy = p.fy[i], fz = p.fz[i];
		const double x0 = p.rx[i], y0 = p.ry[i], z0 = p.rz[i];
		const double vx = __dadd_rn(__dmul_rn(vcorr, vx0), __dmul_rn(a, fx));
		const double vy = __dadd_rn(__dmul_rn(vcorr, vy0), __dmul_rn(a, fy));
		const double vz = __dadd_rn(__dmul_rn(vcorr, vz0), __dmul_rn(a, fz));
		const double x = __dadd_rn(x0, __dmul_rn(dt, vx));
		const double y = __dadd_rn(y0, __dmul_rn(dt, vy));
		const double z = __dadd_rn(z0, __dmul_rn(dt, vz));
		p.vx[i] = vx;
		p.vy[i] = vy;
		p.vz[i] = vz;
		p.rx[i] = x;
		p.ry[i] = y;
		p.rz[i] = z;
		if (sk.flag) {
			const double dx = x - sk.rx[i], dy = y - sk.ry[i], dz = z - sk.rz[i];
			if (!(dx * dx + dy * dy + dz * dz <= sk.half2)) *sk.flag = sk.id;
		}
		if (sk.dmax) {
			// this drift's length squared, rounded up (the bits of a non-negative float order as it does)
			const double sx = x - x0, sy = y - y0, sz = z - z0;
			dm = __float_as_uint(__double2float_ru(sx * sx + sy * sy + sz * sz));
		}
	}
	if (sk.dmax) {
		dm = __reduce_max_sync(0xffffffffu, dm);
		if ((threadIdx.x & 31) == 0 && dm > __ldcg(sk.dmax)) atomicMax(sk.dmax, dm);
	}
}

// Closing kick (Molecule::upd_postF, sum m v^2) of one step, then the opening kick and drift
// (Molecule::upd_preF with vcorr = 1) of the next, with the same roundings as the two kernels.
// Reduction of the block partials inside the kernel (last block) and the step record it completes.
struct Fold {
	unsigned* counter;
	double* out;              // sum m v^2
	const double* scalars;    // U6 sum, virial sum, pair count of the step (from the pair kernel)
	double* record;           // {Upot, virial, sum m v^2, pairs} or null
};

__device__ __forceinline__ void fold(const Fold& f, const double* partials) {
	if (last_block_sum(f.counter, partials, gridDim.x, 1, f.out) && threadIdx.x == 0 && f.record) {
		f.record[0] = f.scalars[0] * 0.5 / 6.;
		f.record[1] = f.scalars[1] * 0.5;
		f.record[2] = f.out[0];
		f.record[3] = f.scalars[2] * 0.5;
	}
}

__global__ void __launch_bounds__(kReduceBlock) k_leapfrog_post_pre(int64_t n, Particles p, SpeciesScale post,
                                                                   SpeciesScale pre, double dt, double* partials,
                                                                   int* status, SkinCheck sk, Fold f) {
	double mv2 = 0.0;
	for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		// every load first: the arrays may alias as far as the compiler knows
		const int t = p.cid[i];
		const double fx = p.fx[i], fy = p.fy[i], fz = p.fz[i];
		const double vx0 = p.vx[i], vy0 = p.vy[i], vz0 = p.vz[i];
		const double x0 = p.rx[i], y0 = p.ry[i], z0 = p.rz[i];
		double rx0 = 0, ry0 = 0, rz0 = 0;
		if (sk.flag) {
			rx0 = sk.rx[i];
			ry0 = sk.ry[i];
			rz0 = sk.rz[i];
		}
		const double a = post.dtInv2m[t];
		const double vx = __dadd_rn(vx0, __dmul_rn(a, fx));
		const double vy = __dadd_rn(vy0, __dmul_rn(a, fy));
		const double vz = __dadd_rn(vz0, __dmul_rn(a, fz));
		const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
		mv2 += __dmul_rn(post.mass[t], v2);
		if (!(v2 == v2) || isinf(v2)) atomicOr(status, kStatusNonFinite);
		const double b = pre.dtInv2m[t];
		const double wx = __dadd_rn(__dmul_rn(1.0, vx), __dmul_rn(b, fx));
		const double wy = __dadd_rn(__dmul_rn(1.0, vy), __dmul_rn(b, fy));
		const double wz = __dadd_rn(__dmul_rn(1.0, vz), __dmul_rn(b, fz));
		const double x = __dadd_rn(x0, __dmul_rn(dt, wx));
		const double y = __dadd_rn(y0, __dmul_rn(dt, wy));
		const double z = __dadd_rn(z0, __dmul_rn(dt, wz));
		p.vx[i] = wx;
		p.vy[i] = wy;
		p.vz[i] = wz;
		p.rx[i] = x;
		p.ry[i] = y;
		p.rz[i] = z;
		if (sk.flag) {
			const double dx = x - rx0, dy = y - ry0, dz = z - rz0;
			if (!(dx * dx + dy * dy + dz * dz <= sk.half2)) *sk.flag = sk.id;
		}
	}
	block_sum3(mv2, 0.0, 0.0, partials);
	fold(f, partials);
}

__global__ void __launch_bounds__(kReduceBlock) k_leapfrog_post(int64_t n, Particles p, SpeciesScale s,
                                                               double* partials, int* status, Fold f) {
	double mv2 = 0.0;
	for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		const int t = p.cid[i];
		const double a = s.dtInv2m[t];
		const double vx0 = p.vx[i], vy0 = p.vy[i], vz0 = p.vz[i];
		const double fx = p.fx[i], fy = p.fy[i], fz = p.fz[i];
		const double vx = __dadd_rn(vx0, __dmul_rn(a, fx));
		const double vy = __dadd_rn(vy0, __dmul_rn(a, fy));
		const double vz = __dadd_rn(vz0, __dmul_rn(a, fz));
		p.vx[i] = vx;
		p.vy[i] = vy;
		p.vz[i] = vz;
		const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
		mv2 += __dmul_rn(s.mass[t], v2);
		if (!(v2 == v2) || isinf(v2)) atomicOr(status, kStatusNonFinite);
	}
	block_sum3(mv2, 0.0, 0.0, partials);
	fold(f, partials);
}

__global__ void k_scale(int64_t n, Particles p, double beta) {
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	p.vx[i] = __dmul_rn(p.vx[i], beta);
	p.vy[i] = __dmul_rn(p.vy[i], beta);
	p.vz[i] = __dmul_rn(p.vz[i], beta);
}

// dst[0..3] = local Upot, local virial, sum m v^2, pair count of the step just finished.
__global__ void k_record(const double* __restrict__ scalars, double* dst) {
	if (threadIdx.x == 0) {
		dst[0] = scalars[0] * 0.5 / 6.;
		dst[1] = scalars[1] * 0.5;
		dst[2] = scalars[3];
		dst[3] = scalars[2] * 0.5;
	}
}

SpeciesScale make_scale(const Context* c, double dt_half) {
	SpeciesScale s{};
	for (int k = 0; k < c->sp.n; k++) {
		s.dtInv2m[k] = dt_half / c->sp.mass[k];
		s.mass[k] = c->sp.mass[k];
	}
	return s;
}

inline unsigned blocks_for(int64_t n) { return (unsigned) ((n + kReduceBlock - 1) / kReduceBlock); }

// Grid of the reducing kernels: the blocks that fit on the device at once (grid-stride loops), so
// that each block's reduction and ticket are paid once per resident block, not per 256 molecules.
template <typename K>
unsigned resident_blocks(const Context* c, K kern, int64_t n) {
	static int per_sm = 0;
	if (per_sm == 0 && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kReduceBlock, 0) != cudaSuccess)
		per_sm = 4;
	const int64_t cap = (int64_t) std::max(per_sm, 1) * c->num_sms;
	return (unsigned) std::max<int64_t>(1, std::min<int64_t>(blocks_for(n), cap));
}

SkinCheck skin_check_of(const Context* c, bool on) {
	SkinCheck sk{};
	if (on) {
		sk.rx = c->r_ref;
		sk.ry = c->r_ref + c->n;
		sk.rz = c->r_ref + 2 * c->n;
		sk.half2 = 0.25 * c->skin * c->skin;
		sk.flag = c->rebuild;
		sk.id = c->step_id;
		if (pruning(c)) sk.dmax = &c->prune_st->dmax[c->step_id & 1];
	}
	return sk;
}

}  // namespace

cudaError_t launch_leapfrog_pre(Context* c, double dt, double vcorr, bool skin_check) {
	if (c->n == 0) return cudaSuccess;
	prof_begin(c, 2);
	const SkinCheck sk = skin_check_of(c, skin_check);
	// dt_halve = .5 * dt, dtInv2m = dt_halve / m  (Molecule.cpp:130-131)
	k_leapfrog_pre<<<blocks_for(c->n), kReduceBlock, 0, c->stream>>>(c->n, c->p, make_scale(c, .5 * dt), dt, vcorr, sk);
	cudaError_t e = cudaGetLastError();
	prof_end(c, 2, 1);
	return e;
}

cudaError_t launch_leapfrog_post_pre(Context* c, double dt, bool skin_check, double* record) {
	prof_begin(c, 2);
	const unsigned nb = resident_blocks(c, k_leapfrog_post_pre, c->n);
	const Fold f{c->tickets + 1, c->scalars + 3, c->scalars, record};
	k_leapfrog_post_pre<<<nb, kReduceBlock, 0, c->stream>>>(
	    c->n, c->p, make_scale(c, 0.5 * dt), make_scale(c, .5 * dt), dt, c->partials, c->status,
	    skin_check_of(c, skin_check), f);
	cudaError_t e = cudaGetLastError();
	prof_end(c, 2, 1);
	return e;
}

cudaError_t launch_leapfrog_post(Context* c, double dt_half, double* record) {
	prof_begin(c, 2);
	const unsigned nb = resident_blocks(c, k_leapfrog_post, c->n);
	const Fold f{c->tickets + 1, c->scalars + 3, c->scalars, record};
	k_leapfrog_post<<<nb, kReduceBlock, 0, c->stream>>>(c->n, c->p, make_scale(c, dt_half), c->partials,
	                                                               c->status, f);
	cudaError_t e = cudaGetLastError();
	prof_end(c, 2, 1);
	return e;
}

cudaError_t launch_scale(Context* c, double beta) {
	if (c->n == 0) return cudaSuccess;
	prof_begin(c, 2);
	k_scale<<<blocks_for(c->n), kReduceBlock, 0, c->stream>>>(c->n, c->p, beta);
	cudaError_t e = cudaGetLastError();
	prof_end(c, 2, 1);
	return e;
}

cudaError_t launch_step_record(Context* c, double* dst) {
	k_record<<<1, 32, 0, c->stream>>>(c->scalars, dst);
	count_launches(c, 1);
	return cudaGetLastError();
}

}  // namespace mdgpu
