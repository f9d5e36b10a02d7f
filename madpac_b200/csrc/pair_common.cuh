// Per-pair arithmetic shared by the pair kernels, and the per-molecule gather over the 27 cells
// around a molecule (used by the simple kernel and as the over-capacity path of the brick kernel).
//
// lj_pair_fp64 follows PotForceLJ (molecules/potforce.h:41-53) and the LJ block of PotForce
// (potforce.h:343-359) operation by operation with round-to-nearest intrinsics (no contraction):
//   invdr2 = 1/dd; lj6 = (sig2*invdr2)^3; lj12 = lj6*lj6; lj12m6 = lj12 - lj6;
//   u = eps24*lj12m6 + shift6; fac = eps24*(lj12 + lj12m6)*invdr2; f = fac*drm;
//   virial term = drm.f.
#pragma once

#include <cuda_runtime.h>

#include "md_internal.h"

namespace mdgpu {

__device__ __forceinline__ void lj_pair_fp64(double d0, double d1, double d2, double dd, double eps24, double sig2,
                                             double shift6, double& f0, double& f1, double& f2, double& u,
                                             double& w) {
	const double invdr2 = __ddiv_rn(1.0, dd);
	double lj6 = __dmul_rn(sig2, invdr2);
	lj6 = __dmul_rn(__dmul_rn(lj6, lj6), lj6);
	const double lj12 = __dmul_rn(lj6, lj6);
	const double lj12m6 = __dsub_rn(lj12, lj6);
	u = __dadd_rn(__dmul_rn(eps24, lj12m6), shift6);
	const double fac = __dmul_rn(__dmul_rn(eps24, __dadd_rn(lj12, lj12m6)), invdr2);
	f0 = __dmul_rn(fac, d0);
	f1 = __dmul_rn(fac, d1);
	f2 = __dmul_rn(fac, d2);
	w = __dadd_rn(__dadd_rn(__dmul_rn(d0, f0), __dmul_rn(d1, f1)), __dmul_rn(d2, f2));
}

struct PairSums {
	double F[3];
	double U, W, np;
	bool same;
};

// Full force on molecule i (sorted index) from all molecules of the 27 cells around its cell.
// params: eps24[ns*ns], sig2 at +kMaxSpecies^2, shift6 at +2*kMaxSpecies^2 (doubles).
template <bool kMixed>
__device__ PairSums gather_pairs(int64_t i, const double* __restrict__ rx, const double* __restrict__ ry,
                                 const double* __restrict__ rz, const int32_t* __restrict__ cid,
                                 const int32_t* __restrict__ start, const Grid& g, const double* params, int ns,
                                 double rc2, double rclj2, int32_t coff = 0) {
	constexpr int KK = kMaxSpecies * kMaxSpecies;
	PairSums s{{0.0, 0.0, 0.0}, 0.0, 0.0, 0.0, false};
	const double xi = rx[i], yi = ry[i], zi = rz[i];
	const int ti = cid[i];
	// cell of i from its position (same formula as the binning)
	int cc[3];
	const double r[3] = {xi, yi, zi};
	for (int d = 0; d < 3; d++) {
		int c = (int) floor(__ddiv_rn(__dsub_rn(r[d], g.halo_min[d]), g.cell_length[d])) - 1;
		cc[d] = c < 0 ? 0 : (c >= g.nc[d] ? g.nc[d] - 1 : c);
	}
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
				const int nb = coff + (z * g.nc[1] + y) * g.nc[0] + x;
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
					s.np += 1.0;
					if (dd == 0.0) s.same = true;
					if (!(dd < rclj2)) continue;
					const int pk = ti * ns + cid[j];
					if (!kMixed) {
						double f0, f1, f2, u, w;
						lj_pair_fp64(d0, d1, d2, dd, params[pk], params[KK + pk], params[2 * KK + pk], f0, f1, f2, u, w);
						s.F[0] += f0;
						s.F[1] += f1;
						s.F[2] += f2;
						s.U += u;
						s.W = __dadd_rn(s.W, w);
					} else {
						const float e0 = (float) d0, e1 = (float) d1, e2 = (float) d2;
						const float ddf = e0 * e0 + e1 * e1 + e2 * e2;
						const float eps24 = (float) params[pk], sig2 = (float) params[KK + pk];
						const float inv = __fdividef(1.0f, ddf);
						const float s2 = sig2 * inv;
						const float s6 = s2 * s2 * s2;
						const float s12 = s6 * s6;
						const float m = s12 - s6;
						const float fac = eps24 * (s12 + m) * inv;
						s.F[0] += (double) (fac * e0);
						s.F[1] += (double) (fac * e1);
						s.F[2] += (double) (fac * e2);
						s.U += (double) (eps24 * m) + params[2 * KK + pk];
						s.W += (double) (fac * ddf);
					}
				}
			}
		}
	}
	return s;
}

}  // namespace mdgpu
