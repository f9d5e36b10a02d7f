// Pair traversal over bricks of 2x2x2 linked cells staged in shared memory.
//
// One CTA (8 warps) owns a brick of 2x2x2 cells; each warp owns one of its cells and computes the
// full force on that cell's molecules from every molecule of the 27 surrounding cells (periodic
// images at +-L, r_j + L / r_j - L as DomainDecompDummy::exchangeMolecules places halo images,
// parallel/DomainDecompDummy.cpp:64-70, 93-99). Per CTA:
//
//  staging  The 4x4x4 cells around the brick are copied to shared memory, ordered by half-cell
//           sub-cells (8x8x8) in x-fastest rows so that any run of sub-cells along x is one
//           contiguous slot range. Positions are stored in a local frame
//           X = x + shift - c_brick + C, C = 1.5 * 2^k with all X of the region in [2^k, 2^(k+1)]:
//           differences of their float "hi" parts are exact (Sterbenz), and a float "lo" part holds
//           X - hi, so (hi_i - hi_j) + (lo_i - lo_j) is X_i - X_j to float rounding. The FP64 mode
//           also stages the double image position x + shift.
//  filter   Each lane (one molecule i) walks only the sub-cells its cutoff sphere can reach (sphere
//           slicing over z, then y, then an x-interval per row), tests r^2 of the hi parts against
//           rc^2 plus a margin that covers the dropped lo parts, and appends hits to its own list.
//  compute  When a list fills (or at the end), every lane evaluates its list: the exact cutoff test
//           (dd < rc^2, strict as BlockTraverse.cpp:155) and PotForceLJ (molecules/potforce.h:41-53)
//           -- in FP64 with the reference's operation order, or in FP32 with FP64 accumulation.
//  fallback A brick whose region holds more molecules than the shared-memory capacity computes
//           its cells by gathering straight from global memory (same per-pair arithmetic).
//
// Each unordered pair is evaluated from both sides; energy and virial are halved on readout.
// Orders of staging, enumeration and accumulation are fixed: results are deterministic.
#include <cuda_runtime.h>

#include <cmath>

#include "md_internal.h"
#include "pair_common.cuh"
#include "reduce.cuh"

namespace mdgpu {
namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kListCap = 64;
constexpr int kSub = 8;              // sub-cells per dimension of the staged region
constexpr int kSubCells = kSub * kSub * kSub;
constexpr unsigned kFull = 0xffffffffu;

struct BrickParams {
	Grid g;
	int nb[3];            // bricks per dimension
	int ns;
	int s_cap;            // staged molecule capacity of the shared-memory layout
	float frame_c[3];     // C per dimension
	float origin[3];      // frame coordinate of the staged region's lower corner
	float h[3], inv_h[3]; // sub-cell width
	float rc2_filter;     // rc^2 + margin covering the lo parts (filter, hi parts only)
	float r_prune;        // sphere radius used to prune sub-cells
	float rc2f, band;     // float rc^2 and the band around it resolved in double
	float rclj2f;
	double rc2, rclj2;
	int lj_is_rc;
};

struct SmemLayout {
	size_t hi, lo, img, sub_start, lists, cell_gid, cell_start, cell_count, cell_k, cell_shift, params, total;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline SmemLayout layout(int s_cap, bool fp64) {
	SmemLayout L;
	size_t o = 0;
	L.hi = o;
	o = align16(o + sizeof(float4) * s_cap);
	L.lo = o;
	if (!fp64) o = align16(o + sizeof(float4) * s_cap);
	L.img = o;
	if (fp64) o = align16(o + sizeof(double) * 3 * s_cap);
	L.sub_start = o;
	o = align16(o + sizeof(int) * (kSubCells + 1));
	L.lists = o;
	o = align16(o + sizeof(unsigned short) * kWarps * kListCap * 32);
	L.cell_gid = o;
	o = align16(o + sizeof(int) * 64);
	L.cell_start = o;
	o = align16(o + sizeof(int) * 64);
	L.cell_count = o;
	o = align16(o + sizeof(int) * 64);
	L.cell_k = o;
	o = align16(o + sizeof(double) * 3 * 64);
	L.cell_shift = o;
	o = align16(o + sizeof(double) * 3 * 64);
	L.params = o;
	o = align16(o + sizeof(double) * 3 * kMaxSpecies * kMaxSpecies + sizeof(float) * 3 * kMaxSpecies * kMaxSpecies);
	L.total = o;
	return L;
}

// sub-cell index (row-major, x fastest) of staged cell (lx, ly, lz) and octant o = ox + 2oy + 4oz
__device__ __forceinline__ int sub_index(int lx, int ly, int lz, int o) {
	return ((2 * lz + ((o >> 2) & 1)) * kSub + (2 * ly + ((o >> 1) & 1))) * kSub + (2 * lx + (o & 1));
}

__device__ __forceinline__ int octant_of(float X, float Y, float Z, int lx, int ly, int lz, const BrickParams& p) {
	const float mx = p.origin[0] + (2 * lx + 1) * p.h[0];
	const float my = p.origin[1] + (2 * ly + 1) * p.h[1];
	const float mz = p.origin[2] + (2 * lz + 1) * p.h[2];
	return (X >= mx ? 1 : 0) | (Y >= my ? 2 : 0) | (Z >= mz ? 4 : 0);
}

template <bool kFP64>
__global__ void __launch_bounds__(kThreads, 2)
    k_pairs_brick(BrickParams p, const double* __restrict__ rx, const double* __restrict__ ry,
                  const double* __restrict__ rz, const int32_t* __restrict__ cid,
                  const int32_t* __restrict__ cstart, const PairParams* __restrict__ pp,
                  double* __restrict__ fx, double* __restrict__ fy, double* __restrict__ fz,
                  double* __restrict__ partials, int* __restrict__ status) {
	extern __shared__ __align__(16) unsigned char smem[];
	const SmemLayout L = layout(p.s_cap, kFP64);
	float4* s_hi = reinterpret_cast<float4*>(smem + L.hi);
	float4* s_lo = reinterpret_cast<float4*>(smem + L.lo);
	double* s_img = reinterpret_cast<double*>(smem + L.img);
	int* s_sub = reinterpret_cast<int*>(smem + L.sub_start);
	unsigned short* s_list = reinterpret_cast<unsigned short*>(smem + L.lists);
	int* s_cgid = reinterpret_cast<int*>(smem + L.cell_gid);
	int* s_cst = reinterpret_cast<int*>(smem + L.cell_start);
	int* s_ccnt = reinterpret_cast<int*>(smem + L.cell_count);
	double* s_ck = reinterpret_cast<double*>(smem + L.cell_k);
	double* s_csh = reinterpret_cast<double*>(smem + L.cell_shift);
	double* s_pd = reinterpret_cast<double*>(smem + L.params);  // eps24, sig2, shift6 (double)
	float* s_pf = reinterpret_cast<float*>(s_pd + 3 * kMaxSpecies * kMaxSpecies);

	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int ns = p.ns;
	const int bx = blockIdx.x % p.nb[0];
	const int by = (blockIdx.x / p.nb[0]) % p.nb[1];
	const int bz = blockIdx.x / (p.nb[0] * p.nb[1]);
	const int bc[3] = {bx, by, bz};

	for (int k = tid; k < ns * ns; k += kThreads) {
		s_pd[k] = pp->eps24[k];
		s_pd[kMaxSpecies * kMaxSpecies + k] = pp->sig2[k];
		s_pd[2 * kMaxSpecies * kMaxSpecies + k] = pp->shift6[k];
		s_pf[k] = (float) pp->eps24[k];
		s_pf[kMaxSpecies * kMaxSpecies + k] = (float) pp->sig2[k];
		s_pf[2 * kMaxSpecies * kMaxSpecies + k] = (float) pp->shift6[k];
	}
	// staged cells: local (lx, ly, lz) in 0..3, global 2b - 1 + l with periodic wrap
	if (tid < 64) {
		const int l[3] = {tid & 3, (tid >> 2) & 3, tid >> 4};
		int gc[3];
		for (int d = 0; d < 3; d++) {
			int gcd = 2 * bc[d] - 1 + l[d];
			double sh = 0.0;
			if (gcd < 0) {
				gcd += p.g.nc[d];
				sh = -p.g.L[d];
			} else if (gcd >= p.g.nc[d]) {
				gcd -= p.g.nc[d];
				sh = p.g.L[d];
			}
			gc[d] = gcd;
			s_csh[3 * tid + d] = sh;
			// frame: X = x + K, K = shift - c_brick + C
			const double cbr = (2 * bc[d] + 1) * p.g.cell_length[d];
			s_ck[3 * tid + d] = (sh - cbr) + (double) p.frame_c[d];
		}
		const int g = (gc[2] * p.g.nc[1] + gc[1]) * p.g.nc[0] + gc[0];
		s_cgid[tid] = g;
		const int st = cstart[g];
		s_cst[tid] = st;
		s_ccnt[tid] = cstart[g + 1] - st;
	}
	for (int k = tid; k < kSubCells + 1; k += kThreads) s_sub[k] = 0;
	__syncthreads();

	// ---- staging pass 1: octant counts of every staged cell ---------------------------------
	for (int c = warp; c < 64; c += kWarps) {
		const int lx = c & 3, ly = (c >> 2) & 3, lz = c >> 4;
		const int st = s_cst[c], cnt = s_ccnt[c];
		const double kx = s_ck[3 * c], ky = s_ck[3 * c + 1], kz = s_ck[3 * c + 2];
		int oc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
		for (int e0 = 0; e0 < cnt; e0 += 32) {
			const int e = e0 + lane;
			int o = -1;
			if (e < cnt) {
				const float X = __double2float_rn(__dadd_rn(rx[st + e], kx));
				const float Y = __double2float_rn(__dadd_rn(ry[st + e], ky));
				const float Z = __double2float_rn(__dadd_rn(rz[st + e], kz));
				o = octant_of(X, Y, Z, lx, ly, lz, p);
			}
#pragma unroll
			for (int q = 0; q < 8; q++) oc[q] += __popc(__ballot_sync(kFull, o == q));
		}
		if (lane < 8) {
			int v = 0;
#pragma unroll
			for (int q = 0; q < 8; q++)
				if (lane == q) v = oc[q];
			s_sub[sub_index(lx, ly, lz, lane)] = v;
		}
	}
	__syncthreads();
	// exclusive scan of the 512 sub-cell counts (2 per thread), total at s_sub[512]
	{
		__shared__ int wsum[kWarps];
		const int a = s_sub[2 * tid], b = s_sub[2 * tid + 1];
		int inc = a + b;
		for (int o = 1; o < 32; o <<= 1) {
			const int y = __shfl_up_sync(kFull, inc, o);
			if (lane >= o) inc += y;
		}
		if (lane == 31) wsum[warp] = inc;
		__syncthreads();
		int off = 0;
		for (int w = 0; w < warp; w++) off += wsum[w];
		const int excl = off + inc - (a + b);
		__syncthreads();
		s_sub[2 * tid] = excl;
		s_sub[2 * tid + 1] = excl + a;
		if (tid == kThreads - 1) s_sub[kSubCells] = excl + a + b;
	}
	__syncthreads();
	const int total = s_sub[kSubCells];
	const bool staged = total <= p.s_cap;

	// ---- staging pass 2: write every molecule to its slot ------------------------------------
	if (staged) {
		for (int c = warp; c < 64; c += kWarps) {
			const int lx = c & 3, ly = (c >> 2) & 3, lz = c >> 4;
			const int st = s_cst[c], cnt = s_ccnt[c];
			const double kx = s_ck[3 * c], ky = s_ck[3 * c + 1], kz = s_ck[3 * c + 2];
			const double shx = s_csh[3 * c], shy = s_csh[3 * c + 1], shz = s_csh[3 * c + 2];
			int base[8] = {0, 0, 0, 0, 0, 0, 0, 0};
			for (int e0 = 0; e0 < cnt; e0 += 32) {
				const int e = e0 + lane;
				int o = -1;
				double x = 0, y = 0, z = 0, Xd = 0, Yd = 0, Zd = 0;
				float X = 0, Y = 0, Z = 0;
				if (e < cnt) {
					x = rx[st + e];
					y = ry[st + e];
					z = rz[st + e];
					Xd = __dadd_rn(x, kx);
					Yd = __dadd_rn(y, ky);
					Zd = __dadd_rn(z, kz);
					X = __double2float_rn(Xd);
					Y = __double2float_rn(Yd);
					Z = __double2float_rn(Zd);
					o = octant_of(X, Y, Z, lx, ly, lz, p);
				}
				const unsigned lt = (1u << lane) - 1u;
				int myoff = 0;
#pragma unroll
				for (int q = 0; q < 8; q++) {
					const unsigned m = __ballot_sync(kFull, o == q);
					if (o == q) myoff = base[q] + __popc(m & lt);
					base[q] += __popc(m);
				}
				if (e < cnt) {
					const int slot = s_sub[sub_index(lx, ly, lz, o)] + myoff;
					const int gi = st + e;
					const int sp = cid[gi];
					s_hi[slot] = make_float4(X, Y, Z, __int_as_float((gi << 3) | sp));
					if (kFP64) {
						s_img[slot] = __dadd_rn(x, shx);
						s_img[p.s_cap + slot] = __dadd_rn(y, shy);
						s_img[2 * p.s_cap + slot] = __dadd_rn(z, shz);
					} else {
						s_lo[slot] = make_float4(__double2float_rn(Xd - (double) X), __double2float_rn(Yd - (double) Y),
						                         __double2float_rn(Zd - (double) Z), 0.f);
					}
				}
			}
		}
	}
	__syncthreads();

	// ---- pairs: warp w owns brick cell (1 + (w&1), 1 + ((w>>1)&1), 1 + (w>>2)) -----------------
	double U = 0.0, W = 0.0, NP = 0.0;
	bool same = false;
	const int il[3] = {1 + (warp & 1), 1 + ((warp >> 1) & 1), 1 + (warp >> 2)};
	const int igc[3] = {2 * bx + il[0] - 1, 2 * by + il[1] - 1, 2 * bz + il[2] - 1};
	const bool cell_ok = igc[0] < p.g.nc[0] && igc[1] < p.g.nc[1] && igc[2] < p.g.nc[2];
	const int icell = il[0] + 4 * il[1] + 16 * il[2];
	if (cell_ok && !staged) {
		// fallback: gather from global memory
		const int st = s_cst[icell], cnt = s_ccnt[icell];
		for (int e = lane; e < cnt; e += 32) {
			PairSums s = gather_pairs<!kFP64>(st + e, rx, ry, rz, cid, cstart, p.g, s_pd, ns, p.rc2, p.rclj2);
			fx[st + e] = s.F[0];
			fy[st + e] = s.F[1];
			fz[st + e] = s.F[2];
			U += s.U;
			W += s.W;
			NP += s.np;
			same |= s.same;
		}
	} else if (cell_ok) {
		// the 8 sub-cells of the i cell and their slot ranges
		int r0[8], rn[8];
		int ni = 0;
#pragma unroll
		for (int o = 0; o < 8; o++) {
			const int sidx = sub_index(il[0], il[1], il[2], o);
			r0[o] = s_sub[sidx];
			rn[o] = s_sub[sidx + 1] - r0[o];
			ni += rn[o];
		}
		unsigned short* mylist = s_list + warp * kListCap * 32 + lane;
		const int nlo[3] = {2 * il[0] - 2, 2 * il[1] - 2, 2 * il[2] - 2};
		const int nhi[3] = {2 * il[0] + 3, 2 * il[1] + 3, 2 * il[2] + 3};
		for (int b0 = 0; b0 < ni; b0 += 32) {
			const int k = b0 + lane;
			const bool act = k < ni;
			int slot_i = 0;
			{
				int acc = 0;
#pragma unroll
				for (int o = 0; o < 8; o++) {
					if (k >= acc && k < acc + rn[o]) slot_i = r0[o] + (k - acc);
					acc += rn[o];
				}
			}
			const float4 hi_i = s_hi[act ? slot_i : 0];
			float4 lo_i = make_float4(0.f, 0.f, 0.f, 0.f);
			double xi = 0, yi = 0, zi = 0;
			if (kFP64) {
				xi = s_img[slot_i];
				yi = s_img[p.s_cap + slot_i];
				zi = s_img[2 * p.s_cap + slot_i];
			} else {
				lo_i = s_lo[slot_i];
			}
			const int ti = __float_as_int(hi_i.w) & 7;
			const int gi = __float_as_int(hi_i.w) >> 3;
			// enumeration state: z slices, y rows, x interval of sub-cells
			const float R = p.r_prune, R2 = R * R;
			int sz = 0, sz_hi = -1, sy = 0, sy_hi = -1;
			float rem_z = 0.f;
			if (act) {
				sz = max(nlo[2], (int) floorf((hi_i.z - R - p.origin[2]) * p.inv_h[2]));
				sz_hi = min(nhi[2], (int) floorf((hi_i.z + R - p.origin[2]) * p.inv_h[2]));
				sz -= 1;
			}
			int pp_ = 0, pe_ = 0;
			bool done = !act;
			int cnt = 0;
			double Fx = 0.0, Fy = 0.0, Fz = 0.0;
			auto flush = [&]() {
				const int mx = __reduce_max_sync(kFull, cnt);
				float ax = 0.f, ay = 0.f, az = 0.f, au = 0.f, aw = 0.f;
				double dx64 = 0, dy64 = 0, dz64 = 0, du64 = 0, dw64 = 0;
				int anp = 0;
				for (int t = 0; t < mx; t++) {
					if (t >= cnt) continue;
					const int j = mylist[t * 32];
					const float4 hj = s_hi[j];
					const int pk = ti * ns + (__float_as_int(hj.w) & 7);
					if (kFP64) {
						const double d0 = __dsub_rn(xi, s_img[j]);
						const double d1 = __dsub_rn(yi, s_img[p.s_cap + j]);
						const double d2 = __dsub_rn(zi, s_img[2 * p.s_cap + j]);
						const double dd = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
						if (!(dd < p.rc2)) continue;
						anp++;
						if (dd == 0.0) same = true;
						if (!(dd < p.rclj2)) continue;
						double f0, f1, f2, u, w;
						lj_pair_fp64(d0, d1, d2, dd, s_pd[pk], s_pd[kMaxSpecies * kMaxSpecies + pk],
						             s_pd[2 * kMaxSpecies * kMaxSpecies + pk], f0, f1, f2, u, w);
						dx64 += f0;
						dy64 += f1;
						dz64 += f2;
						du64 += u;
						dw64 = __dadd_rn(dw64, w);
					} else {
						const float4 lj = s_lo[j];
						const float h0 = hi_i.x - hj.x, h1 = hi_i.y - hj.y, h2 = hi_i.z - hj.z;  // exact
						const float l0 = lo_i.x - lj.x, l1 = lo_i.y - lj.y, l2 = lo_i.z - lj.z;
						const float e0 = h0 + l0, e1 = h1 + l1, e2 = h2 + l2;
						const float d2f = fmaf(e0, e0, fmaf(e1, e1, e2 * e2));
						bool in;
						if (fabsf(d2f - p.rc2f) <= p.band) {
							const double a0 = (double) h0 + ((double) lo_i.x - (double) lj.x);
							const double a1 = (double) h1 + ((double) lo_i.y - (double) lj.y);
							const double a2 = (double) h2 + ((double) lo_i.z - (double) lj.z);
							in = a0 * a0 + a1 * a1 + a2 * a2 < p.rc2;
						} else {
							in = d2f < p.rc2f;
						}
						if (!in) continue;
						anp++;
						if (d2f == 0.f) same = true;
						if (!p.lj_is_rc && !(d2f < p.rclj2f)) continue;
						const float eps24 = s_pf[pk], sig2 = s_pf[kMaxSpecies * kMaxSpecies + pk];
						const float inv = __fdividef(1.0f, d2f);
						const float s2 = sig2 * inv;
						const float s6 = s2 * s2 * s2;
						const float s12 = s6 * s6;
						const float m = s12 - s6;
						const float fac = eps24 * (s12 + m) * inv;
						ax = fmaf(fac, e0, ax);
						ay = fmaf(fac, e1, ay);
						az = fmaf(fac, e2, az);
						au += fmaf(eps24, m, s_pf[2 * kMaxSpecies * kMaxSpecies + pk]);
						aw = fmaf(fac, d2f, aw);
					}
				}
				if (kFP64) {
					Fx += dx64;
					Fy += dy64;
					Fz += dz64;
					U += du64;
					W += dw64;
				} else {
					Fx += (double) ax;
					Fy += (double) ay;
					Fz += (double) az;
					U += (double) au;
					W += (double) aw;
				}
				NP += (double) anp;
				cnt = 0;
			};
			while (true) {
				// advance to the next non-empty run of candidate slots
				while (pp_ == pe_ && !done) {
					if (sy < sy_hi) {
						++sy;
						const float y0 = p.origin[1] + sy * p.h[1];
						const float gy = fmaxf(0.f, fmaxf(y0 - hi_i.y, hi_i.y - (y0 + p.h[1])));
						const float rem = rem_z - gy * gy;
						if (rem > 0.f) {
							const float wx = sqrtf(rem);
							const int sxl = max(nlo[0], (int) floorf((hi_i.x - wx - p.origin[0]) * p.inv_h[0]));
							const int sxh = min(nhi[0], (int) floorf((hi_i.x + wx - p.origin[0]) * p.inv_h[0]));
							if (sxl <= sxh) {
								const int row = (sz * kSub + sy) * kSub;
								pp_ = s_sub[row + sxl];
								pe_ = s_sub[row + sxh + 1];
							}
						}
					} else {
						++sz;
						if (sz > sz_hi) {
							done = true;
						} else {
							const float z0 = p.origin[2] + sz * p.h[2];
							const float gz = fmaxf(0.f, fmaxf(z0 - hi_i.z, hi_i.z - (z0 + p.h[2])));
							rem_z = R2 - gz * gz;
							if (rem_z > 0.f) {
								const float wy = sqrtf(rem_z);
								sy = max(nlo[1], (int) floorf((hi_i.y - wy - p.origin[1]) * p.inv_h[1])) - 1;
								sy_hi = min(nhi[1], (int) floorf((hi_i.y + wy - p.origin[1]) * p.inv_h[1]));
							} else {
								sy = 0;
								sy_hi = -1;
							}
						}
					}
				}
				const bool has = pp_ < pe_;
				if (!__any_sync(kFull, has)) break;
				if (has) {
					const int j = pp_++;
					const float4 hj = s_hi[j];
					const float d0 = hi_i.x - hj.x, d1 = hi_i.y - hj.y, d2 = hi_i.z - hj.z;
					const float dd = fmaf(d0, d0, fmaf(d1, d1, d2 * d2));
					if (dd < p.rc2_filter && j != slot_i) {
						mylist[cnt * 32] = (unsigned short) j;
						cnt++;
					}
				}
				if (__any_sync(kFull, cnt == kListCap)) flush();
			}
			flush();
			if (act) {
				fx[gi] = Fx;
				fy[gi] = Fy;
				fz[gi] = Fz;
				if (!(Fx == Fx && Fy == Fy && Fz == Fz) || isinf(Fx) || isinf(Fy) || isinf(Fz))
					atomicOr(status, kStatusNonFinite);
			}
		}
	}
	if (same) atomicOr(status, kStatusSamePosition);
	block_sum3(U, W, NP, partials);
}

}  // namespace

cudaError_t launch_pairs_brick(Context* c) {
	const bool fp64 = c->precision == MDGPU_FP64;
	BrickParams p{};
	p.g = c->g;
	p.ns = c->sp.n;
	for (int d = 0; d < 3; d++) {
		p.nb[d] = (c->g.nc[d] + 1) / 2;
		const double cl = c->g.cell_length[d];
		// smallest 2^k with the staged region X in [C - 2cl, C + 2cl] inside [2^k, 2^(k+1)]
		double pk = 1.0;
		while (pk < 4.0 * cl) pk *= 2.0;
		p.frame_c[d] = (float) (1.5 * pk);
		p.origin[d] = (float) (1.5 * pk - 2.0 * cl);
		p.h[d] = (float) (0.5 * cl);
		p.inv_h[d] = (float) (1.0 / (0.5 * cl));
	}
	double ulp = 0;  // largest float ulp of a frame coordinate
	for (int d = 0; d < 3; d++) {
		double u = std::ldexp(1.0, std::ilogb((double) p.frame_c[d] + 2.0 * c->g.cell_length[d]) - 23);
		ulp = u > ulp ? u : ulp;
	}
	const double rc = c->rc;
	p.rc2 = rc * rc;
	p.rclj2 = c->rc_lj * c->rc_lj;
	p.rc2f = (float) p.rc2;
	p.rclj2f = (float) p.rclj2;
	p.lj_is_rc = c->rc_lj == c->rc;
	// the dropped lo parts move each coordinate difference by < 1 ulp; grow the radius by 4 ulp
	p.rc2_filter = (float) ((rc + 4.0 * ulp * 1.7320508) * (rc + 4.0 * ulp * 1.7320508) + 1e-6 * p.rc2);
	p.r_prune = (float) (rc + 8.0 * ulp * 1.7320508 + 1e-5 * rc);
	p.band = (float) (4e-6 * p.rc2);

	// shared-memory capacity: two CTAs per SM
	static int max_optin = -1;
	if (max_optin < 0) cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
	const size_t budget = 110 * 1024;
	int s_cap = 256;
	while (layout(s_cap + 64, fp64).total <= budget && layout(s_cap + 64, fp64).total <= (size_t) max_optin) s_cap += 64;
	if (s_cap > 65535) s_cap = 65535;
	p.s_cap = s_cap;
	const size_t bytes = layout(s_cap, fp64).total;
	const int nbricks = p.nb[0] * p.nb[1] * p.nb[2];
	prof_begin(c, 1);
	cudaError_t e;
	if (fp64) {
		e = cudaFuncSetAttribute(k_pairs_brick<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bytes);
		if (e == cudaSuccess)
			k_pairs_brick<true><<<nbricks, kThreads, bytes, c->stream>>>(p, c->p.rx, c->p.ry, c->p.rz, c->p.cid,
			                                                             c->cell_start, c->d_pp, c->p.fx, c->p.fy,
			                                                             c->p.fz, c->partials, c->status);
	} else {
		e = cudaFuncSetAttribute(k_pairs_brick<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bytes);
		if (e == cudaSuccess)
			k_pairs_brick<false><<<nbricks, kThreads, bytes, c->stream>>>(p, c->p.rx, c->p.ry, c->p.rz, c->p.cid,
			                                                              c->cell_start, c->d_pp, c->p.fx, c->p.fy,
			                                                              c->p.fz, c->partials, c->status);
	}
	if (e == cudaSuccess) e = cudaGetLastError();
	prof_end(c, 1, 1);
	if (e != cudaSuccess) return e;
	return launch_reduce(c, nbricks, c->scalars, 3);
}

}  // namespace mdgpu
