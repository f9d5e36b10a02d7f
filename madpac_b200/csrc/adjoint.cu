// Adjoint (vector-Jacobian product) of the LJ forces and potential energy.
//
// For a loss L whose cotangents are gF_i = dL/dF_i and gU = dL/dUpot, this kernel returns
// dL/dr_k and dL/d(eps_ab), dL/d(sigma_ab) for every component pair, where the pair parameters are
// eps_ab = eps24/24 and sigma_ab = sqrt(sig2) of the Comp2Param stream (Comp2Param.cpp:28-115;
// paths relative to madpac/mardyn/). The reference has no gradients; the forward quantities are
// those of PotForceLJ (molecules/potforce.h:41-53) with Upot = sum (u6 + shift6)/6
// (ParticlePairs2PotForceAdapter.h:65).
//
// Per pair, d = r_i - r_j, q = d.d, s6 = (sig2/q)^3, s12 = s6^2:
//   f = fac d,  fac = eps24 (2 s12 - s6)/q,  dfac/dq = eps24 (4 s6 - 14 s12)/q^2
//   J = df/dd = fac I + 2 dfac/dq d d^T   (symmetric),   dU_pair/dd = -f
//   dL/dr_i += J (gF_i - gF_j) - gU f
//   df/deps24 = f/eps24;  df/dsig2 = eps24 (12 s12 - 3 s6)/(q sig2) d
//   dU_pair/deps24 = (s12 - s6 + c6)/6,  dU_pair/dsig2 = eps24 (6 s12 - 3 s6 + c6')/(6 sig2)
// with c6 = sr6 - sr6^2, c6' = 3 sr6 - 6 sr6^2 (sr6 = (sig2/rcLJ^2)^3) for truncated-shifted pair
// types (shift6 != 0) and 0 otherwise. Every molecule gathers over its 27 neighbour cells (each
// pair is seen from both sides, so parameter terms carry a factor 1/2; kAdjLanes lanes share a
// molecule's candidates and sum their parts by a fixed butterfly). FP64 throughout, or (the
// mixed form, MDGPU_MIXED) the pair's derivative terms in FP32 from the FP64 difference vector,
// with the cutoff decided in FP64 and every sum kept in FP64. The parameter terms are summed per
// block in a fixed order (per-warp partials, then warp by warp), so the results do not depend on
// scheduling.
#include <cuda_runtime.h>

#include "md_internal.h"
#include "reduce.cuh"

namespace mdgpu {
namespace {

constexpr int KK = kMaxSpecies * kMaxSpecies;
constexpr int kAdjList = 16;   // accepted partners a lane lists before evaluating them

// NP: the number of species pairs held in registers (ns * ns, 1 or 4), or 0 for any ns up to
// kMaxSpecies with the per-pair sums in a KK-entry array (local memory).
template <bool kMixed, int NP>
__global__ void __launch_bounds__(kReduceBlock) k_adjoint(int64_t n, Particles p, const int32_t* __restrict__ start,
                                                         Grid g, const PairParams* __restrict__ pp, double rclj,
                                                         const double* __restrict__ gfx, const double* __restrict__ gfy,
                                                         const double* __restrict__ gfz, double gU,
                                                         double* __restrict__ ox, double* __restrict__ oy,
                                                         double* __restrict__ oz, double* __restrict__ pgrad) {
	__shared__ double s_e24[KK], s_s2[KK], s_sh[KK];
	__shared__ double s_acc[kReduceBlock / 32][2 * KK];   // per-warp partials of the parameter terms
	__shared__ int32_t s_aj[kAdjList * kReduceBlock];      // each lane's accepted partners (column per lane)
	__shared__ uint8_t s_ai[kAdjList * kReduceBlock];      // and their periodic images (27 codes)
	const int ns = pp->ns;
	for (int k = threadIdx.x; k < KK; k += blockDim.x) {
		s_e24[k] = k < ns * ns ? pp->eps24[k] : 0.0;
		s_s2[k] = k < ns * ns ? pp->sig2[k] : 0.0;
		s_sh[k] = k < ns * ns ? pp->shift6[k] : 0.0;
	}
	__syncthreads();
	const double rc2 = pp->rc2, rclj2 = pp->rclj2, rclj6 = rclj2 * rclj2 * rclj2;
	// kAdjLanes consecutive lanes per molecule, each taking every kAdjLanes-th candidate of a cell
	const int64_t i = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) / kAdjLanes;
	const int sub = threadIdx.x % kAdjLanes;
	constexpr int NA = NP > 0 ? NP : KK;
	double acc_e[NA], acc_s[NA];
#pragma unroll
	for (int k = 0; k < NA; k++) acc_e[k] = acc_s[k] = 0.0;
	// adds to the sums of species pair pk (with NP > 0 by selection, so the sums stay in registers)
	auto add_param = [&](int pk, double ve, double vs) {
		if constexpr (NP > 0) {
#pragma unroll
			for (int k = 0; k < NP; k++)
				if (k == pk) {
					acc_e[k] += ve;
					acc_s[k] += vs;
				}
		} else {
			acc_e[pk] += ve;
			acc_s[pk] += vs;
		}
	};
	double ax = 0.0, ay = 0.0, az = 0.0;
	if (i < n) {
		const double xi = p.rx[i], yi = p.ry[i], zi = p.rz[i];
		const double wix = gfx[i], wiy = gfy[i], wiz = gfz[i];
		const int ti = p.cid[i];
		int cc[3];
		const double r[3] = {xi, yi, zi};
		for (int d = 0; d < 3; d++) {
			int c = (int) floor(__ddiv_rn(__dsub_rn(r[d], g.halo_min[d]), g.cell_length[d])) - 1;
			cc[d] = c < 0 ? 0 : (c >= g.nc[d] ? g.nc[d] - 1 : c);
		}
		// accepted partners are listed per lane and evaluated together, so that the lanes of a warp run
		// the pair VJP side by side (each lane in the order it accepted them, as it would inline)
		uint32_t acnt = 0;
		int32_t* aj = s_aj + threadIdx.x;
		uint8_t* ai = s_ai + threadIdx.x;
		auto eval_pair = [&](int j, double sx, double sy, double sz) {
			const double d0 = xi - (p.rx[j] + sx), d1 = yi - (p.ry[j] + sy), d2 = zi - (p.rz[j] + sz);
			const double q = d0 * d0 + d1 * d1 + d2 * d2;
			const int pk = ti * ns + p.cid[j];
			const double e24 = s_e24[pk], sg2 = s_s2[pk];
			const double w0 = wix - gfx[j], w1 = wiy - gfy[j], w2 = wiz - gfz[j];
			const bool shf = s_sh[pk] != 0.0;
			const double sr6 = sg2 * sg2 * sg2 / rclj6;
			const double c6 = shf ? sr6 - sr6 * sr6 : 0.0;
			const double c6s = shf ? 3.0 * sr6 - 6.0 * sr6 * sr6 : 0.0;
			if (kMixed) {
				// FP32 from the FP64 difference vector; FP64 sums
				const float f0 = (float) d0, f1 = (float) d1, f2 = (float) d2;
				const float qf = fmaf(f0, f0, fmaf(f1, f1, f2 * f2));
				const float e24f = (float) e24, sg2f = (float) sg2;
				const float iq = 1.0f / qf;
				float s6 = sg2f * iq;
				s6 = s6 * s6 * s6;
				const float s12 = s6 * s6;
				const float fac = e24f * (2.0f * s12 - s6) * iq;
				const float dfac = e24f * (4.0f * s6 - 14.0f * s12) * iq * iq;
				const float v0 = (float) w0, v1 = (float) w1, v2 = (float) w2;
				const float dw = fmaf(f0, v0, fmaf(f1, v1, f2 * v2));
				const float gUf = (float) gU;
				const float t = 2.0f * dfac * dw;
				ax += (double) (fac * v0 + t * f0 - gUf * fac * f0);
				ay += (double) (fac * v1 + t * f1 - gUf * fac * f1);
				az += (double) (fac * v2 + t * f2 - gUf * fac * f2);
				add_param(pk, 0.5 * ((double) (fac * dw / e24f) + gU * ((double) (s12 - s6) + c6) / 6.0),
				          0.5 * ((double) (e24f * (12.0f * s12 - 3.0f * s6) * iq / sg2f * dw) +
				                 gU * e24 * ((double) (6.0f * s12 - 3.0f * s6) + c6s) / (6.0 * sg2)));
			} else {
				const double iq = 1.0 / q;
				double s6 = sg2 * iq;
				s6 = s6 * s6 * s6;
				const double s12 = s6 * s6;
				const double fac = e24 * (2.0 * s12 - s6) * iq;
				const double dfac = e24 * (4.0 * s6 - 14.0 * s12) * iq * iq;
				const double dw = d0 * w0 + d1 * w1 + d2 * w2;
				// J w - gU f
				ax += fac * w0 + 2.0 * dfac * dw * d0 - gU * fac * d0;
				ay += fac * w1 + 2.0 * dfac * dw * d1 - gU * fac * d1;
				az += fac * w2 + 2.0 * dfac * dw * d2 - gU * fac * d2;
				// parameter terms (half: the pair is seen from both sides)
				add_param(pk, 0.5 * (fac * dw / e24 + gU * (s12 - s6 + c6) / 6.0),
				          0.5 * (e24 * (12.0 * s12 - 3.0 * s6) * iq / sg2 * dw +
				                 gU * e24 * (6.0 * s12 - 3.0 * s6 + c6s) / (6.0 * sg2)));
			}
		};
		auto flush = [&]() {
			for (uint32_t e = 0; e < acnt; e++) {
				const int j = aj[e * kReduceBlock];
				const int img = ai[e * kReduceBlock];
				eval_pair(j, (double) (img % 3 - 1) * g.L[0], (double) ((img / 3) % 3 - 1) * g.L[1],
				          (double) (img / 9 - 1) * g.L[2]);
			}
			acnt = 0;
		};
		for (int dz = -1; dz <= 1; dz++) {
			int z = cc[2] + dz;
			double sz = 0.0;
			if (z < 0) {
				z += g.nc[2];
				sz = -g.L[2];
			} else if (z >= g.nc[2]) {
				z -= g.nc[2];
				sz = g.L[2];
			}
			for (int dy = -1; dy <= 1; dy++) {
				int y = cc[1] + dy;
				double sy = 0.0;
				if (y < 0) {
					y += g.nc[1];
					sy = -g.L[1];
				} else if (y >= g.nc[1]) {
					y -= g.nc[1];
					sy = g.L[1];
				}
				for (int dx = -1; dx <= 1; dx++) {
					int x = cc[0] + dx;
					double sx = 0.0;
					if (x < 0) {
						x += g.nc[0];
						sx = -g.L[0];
					} else if (x >= g.nc[0]) {
						x -= g.nc[0];
						sx = g.L[0];
					}
					const int nb = (z * g.nc[1] + y) * g.nc[0] + x;
					const bool shifted = (sx != 0.0) || (sy != 0.0) || (sz != 0.0);
					const uint8_t img = (uint8_t) ((sx < 0.0 ? 0 : sx > 0.0 ? 2 : 1) + 3 * (sy < 0.0 ? 0 : sy > 0.0 ? 2 : 1) +
					                               9 * (sz < 0.0 ? 0 : sz > 0.0 ? 2 : 1));
					for (int j = start[nb] + sub; j < start[nb + 1]; j += kAdjLanes) {
						if (j == i && !shifted) continue;
						const double d0 = xi - (p.rx[j] + sx), d1 = yi - (p.ry[j] + sy), d2 = zi - (p.rz[j] + sz);
						const double q = d0 * d0 + d1 * d1 + d2 * d2;
						if (!(q < rc2) || !(q < rclj2)) continue;
						aj[acnt * kReduceBlock] = j;
						ai[acnt * kReduceBlock] = img;
						if (++acnt == kAdjList) flush();
					}
				}
			}
		}
		flush();
	}
	// the molecule's lanes' sums in a fixed order
	for (int o = 1; o < kAdjLanes; o <<= 1) {
		ax += __shfl_xor_sync(0xffffffffu, ax, o);
		ay += __shfl_xor_sync(0xffffffffu, ay, o);
		az += __shfl_xor_sync(0xffffffffu, az, o);
	}
	if (i < n && sub == 0) {
		ox[i] = ax;
		oy[i] = ay;
		oz[i] = az;
	}
	// block sum of the per-type parameter terms in a fixed order (warp sums, then warp by warp),
	// then one partial row per block
	const int warp = threadIdx.x >> 5;
#pragma unroll
	for (int k = 0; k < NA; k++) {
		if (NP == 0 && k >= ns * ns) break;   // warp-uniform
		const double ve = warp_sum(acc_e[k]), vs = warp_sum(acc_s[k]);
		if ((threadIdx.x & 31) == 0) {
			s_acc[warp][k] = ve;
			s_acc[warp][KK + k] = vs;
		}
	}
	if ((threadIdx.x & 31) == 0)
		for (int k = ns * ns; k < KK; k++) s_acc[warp][k] = s_acc[warp][KK + k] = 0.0;
	__syncthreads();
	for (int k = threadIdx.x; k < 2 * KK; k += blockDim.x) {
		double v = 0.0;
		for (int w = 0; w < kReduceBlock / 32; w++) v += s_acc[w][k];
		pgrad[(int64_t) blockIdx.x * 2 * KK + k] = v;
	}
}

// Sum of the blocks' rows into out (added to it with `accumulate`), in a fixed order: one block of
// kParamGroups x 2 KK threads; group q sums rows q, q + kParamGroups, ... (each load of a group is
// one contiguous row), then the groups' sums are added in group order.
constexpr int kParamGroups = 8;
__global__ void __launch_bounds__(kParamGroups * 2 * KK) k_adjoint_params(int64_t nblocks,
                                                                          const double* __restrict__ pgrad,
                                                                          double* __restrict__ out, bool accumulate) {
	__shared__ double s_part[kParamGroups][2 * KK];
	const int k = threadIdx.x % (2 * KK), q = threadIdx.x / (2 * KK);
	double s = 0.0;
	for (int64_t b = q; b < nblocks; b += kParamGroups) s += pgrad[b * 2 * KK + k];
	s_part[q][k] = s;
	__syncthreads();
	if (q == 0) {
		double t = s_part[0][k];
		for (int g = 1; g < kParamGroups; g++) t += s_part[g][k];
		out[k] = accumulate ? out[k] + t : t;
	}
}

}  // namespace

cudaError_t launch_adjoint(Context* c, const double* gfx, const double* gfy, const double* gfz, double gU, double* ox,
                           double* oy, double* oz, double* pgrad, double* pout, bool accumulate) {
	const int64_t nb = adjoint_blocks(c->n);
	const int np = c->sp.n * c->sp.n;
#define MD_ADJ(MX, NPV)                                                                                           \
	k_adjoint<MX, NPV><<<(unsigned) nb, kReduceBlock, 0, c->stream>>>(c->n, c->p, c->cell_start, c->g, c->d_pp,   \
	                                                                   c->rc_lj, gfx, gfy, gfz, gU, ox, oy, oz, pgrad)
	const bool mixed = c->precision == MDGPU_MIXED;
	if (np == 1)
		mixed ? MD_ADJ(true, 1) : MD_ADJ(false, 1);
	else if (np == 4)
		mixed ? MD_ADJ(true, 4) : MD_ADJ(false, 4);
	else
		mixed ? MD_ADJ(true, 0) : MD_ADJ(false, 0);
#undef MD_ADJ
	k_adjoint_params<<<1, kParamGroups * 2 * KK, 0, c->stream>>>(nb, pgrad, pout, accumulate);
	count_launches(c, 2);
	return cudaGetLastError();
}

}  // namespace mdgpu
