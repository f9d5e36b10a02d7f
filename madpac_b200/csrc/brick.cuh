// Pair traversal of one brick of 2x2x2 linked cells staged in shared memory (device function used
// by the single-box pair kernel and by the persistent multi-box step kernel).
//
// One CTA (8 warps) owns a brick of 2x2x2 cells; each warp owns one of its cells and computes the
// full force on that cell's molecules from every molecule of the 27 surrounding cells (periodic
// images at +-L, r_j + L / r_j - L as DomainDecompDummy::exchangeMolecules places halo images,
// parallel/DomainDecompDummy.cpp:64-70, 93-99; paths relative to madpac/mardyn/). Per brick:
//
//  staging  The 4x4x4 cells around the brick are copied to shared memory cell by cell (x fastest),
//           so the 3 cells of each neighbour row of a cell form one contiguous slot range.
//           Positions are stored in a local frame
//           X = x + shift - c_brick + C, C = 1.5 * 2^k with all X of the region in [2^k, 2^(k+1)]:
//           differences of their float "hi" parts are exact (Sterbenz), and a float "lo" part holds
//           X - hi, so (hi_i - hi_j) + (lo_i - lo_j) is X_i - X_j to float rounding. The FP64 mode
//           also stages the double image position x + shift.
//  filter   Each lane holds one molecule i; every pair of consecutive staged molecules j of the 9
//           neighbour rows is broadcast to all lanes, which test r^2 in packed half precision
//           against rc^2 plus a margin covering the rounding, and append hits to their own list.
//  compute  When a list fills (or at the end), every lane evaluates its list: the exact cutoff test
//           (dd < rc^2, strict as BlockTraverse.cpp:155) and PotForceLJ (molecules/potforce.h:41-53)
//           -- in FP64 with the reference's operation order, or in FP32 with FP64 accumulation.
//  fallback A brick whose region holds more molecules than the shared-memory capacity computes
//           its cells by gathering straight from global memory (same per-pair arithmetic).
//
// Each unordered pair is evaluated from both sides; energy and virial are halved on readout.
// Orders of staging, enumeration and accumulation are fixed: results are deterministic and do not
// depend on which CTA evaluates a brick.
#pragma once

#include <cuda_runtime.h>

#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>

#include "md_internal.h"
#include "pair_common.cuh"
#include "reduce.cuh"

namespace mdgpu {
namespace brick {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr unsigned kFull = 0xffffffffu;
constexpr int KK = kMaxSpecies * kMaxSpecies;

// Constants shared by every brick of a launch.
struct Const {
	int ns;
	int s_cap;            // staged molecule capacity of the shared-memory layout
	float rc2f, band;     // float rc^2 and the band around it resolved in double
	float rclj2f;
	double rc2, rclj2;
};

// One periodic box as the brick code sees it: its cell grid, its bricks per dimension, the offset of
// its cells in the cell-start array, and the frame constants of the packed filter.
struct Box {
	Grid g;
	int nb[3];
	int32_t coff;
	float frame_c[3];     // C per dimension
	float rc2_h;          // rc^2 + margin covering half-precision rounding (packed filter)
};

struct SmemLayout {
	size_t hi, lo, img, h16, cstart, lists, ccount, gstart, cell_k, cell_shift, params, total;
};

// Two consecutive staged molecules in half precision, relative to the brick centre: the packed
// filter tests two candidates per instruction.
struct __align__(16) HalfPair {
	__half2 x, y, z, pad;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline SmemLayout layout(int s_cap, bool fp64, int list_cap) {
	SmemLayout L;
	size_t o = 0;
	L.hi = o;
	o = align16(o + sizeof(float4) * s_cap);
	L.lo = o;
	if (!fp64) o = align16(o + sizeof(float4) * s_cap);
	L.img = o;
	if (fp64) o = align16(o + sizeof(double) * 3 * s_cap);
	L.h16 = o;
	o = align16(o + sizeof(HalfPair) * (s_cap / 2 + 20));  // 32-slot blocks may read past the end
	L.cstart = o;
	o = align16(o + sizeof(int) * 65);
	L.lists = o;
	o = align16(o + sizeof(unsigned short) * kWarps * list_cap * 32);
	L.ccount = o;
	o = align16(o + sizeof(int) * 64);
	L.gstart = o;
	o = align16(o + sizeof(int) * 64);
	L.cell_k = o;
	o = align16(o + sizeof(double) * 3 * 64);
	L.cell_shift = o;
	o = align16(o + sizeof(double) * 3 * 64);
	L.params = o;
	o = align16(o + sizeof(double) * 3 * KK + sizeof(float) * 3 * KK);
	L.total = o;
	return L;
}

// Largest staged capacity (a multiple of 64) whose layout fits in `budget` bytes.
inline int capacity_for(size_t budget, bool fp64, int list_cap) {
	int s_cap = 256;
	while (layout(s_cap + 64, fp64, list_cap).total <= budget) s_cap += 64;
	return s_cap > 65535 ? 65535 : s_cap;
}

// Frame constants of one box (host side).
inline void init_box(Box& b, const Grid& g, double rc, int32_t coff) {
	b.g = g;
	b.coff = coff;
	for (int d = 0; d < 3; d++) {
		b.nb[d] = (g.nc[d] + 1) / 2;
		const double cl = g.cell_length[d];
		// smallest 2^k with the staged region X in [C - 2cl, C + 2cl] inside [2^k, 2^(k+1)]
		double pk = 1.0;
		while (pk < 4.0 * cl) pk *= 2.0;
		b.frame_c[d] = (float) (1.5 * pk);
	}
	// half-precision filter: coordinates within +-2 cells of the brick centre; each rounding is at
	// most half an ulp of the largest coordinate, plus the rounding of the packed r^2 itself
	const double cmax = 2.0 * std::max(g.cell_length[0], std::max(g.cell_length[1], g.cell_length[2]));
	const double uc = std::ldexp(1.0, std::ilogb(cmax) - 10);   // half ulp at cmax (10-bit mantissa)
	const double du = 2.0 * uc * 1.7320508;                     // |error of the difference vector|
	const double r2max = (rc + du) * (rc + du);
	const double ur2 = std::ldexp(1.0, std::ilogb(r2max) - 10);
	b.rc2_h = (float) (r2max + 4.0 * ur2 + 1e-3);
}

inline Const make_const(int ns, int s_cap, double rc, double rc_lj) {
	Const p{};
	p.ns = ns;
	p.s_cap = s_cap;
	p.rc2 = rc * rc;
	p.rclj2 = rc_lj * rc_lj;
	p.rc2f = (float) p.rc2;
	p.rclj2f = (float) p.rclj2;
	p.band = (float) (4e-6 * p.rc2);
	return p;
}

// Reciprocal by the hardware approximation (rcp.approx.ftz.f32, about 1 ulp).
__device__ __forceinline__ float rcp_approx(float x) {
	float r;
	asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
	return r;
}

// Copies the Comp2Param table to shared memory (double and float); the caller synchronises.
__device__ __forceinline__ void load_params(unsigned char* smem, const SmemLayout& L, const PairParams* pp, int ns) {
	double* s_pd = reinterpret_cast<double*>(smem + L.params);
	float* s_pf = reinterpret_cast<float*>(s_pd + 3 * KK);
	for (int k = threadIdx.x; k < ns * ns; k += kThreads) {
		s_pd[k] = pp->eps24[k];
		s_pd[KK + k] = pp->sig2[k];
		s_pd[2 * KK + k] = pp->shift6[k];
		s_pf[k] = (float) pp->eps24[k];
		s_pf[KK + k] = (float) pp->sig2[k];
		s_pf[2 * KK + k] = (float) pp->shift6[k];
	}
}

// Forces on the molecules of brick `brick` (index within its box) of box `bx`; U, W and the pair
// count go to partials[slot]. The pair table must already be in shared memory (load_params).
// Ends with a CTA-wide barrier after which no thread reads the staged data.
template <bool kFP64, bool kSingle, bool kLjIsRc, int kCap>
__device__ __forceinline__ void pairs(const Const& p, const Box& bx, int brick, int64_t slot, unsigned char* smem,
                                      const double* rx, const double* ry, const double* rz, const int32_t* cid,
                                      const int32_t* cstart, double* fx, double* fy, double* fz, double* partials,
                                      int* status) {
	const SmemLayout L = layout(p.s_cap, kFP64, kCap);
	float4* s_hi = reinterpret_cast<float4*>(smem + L.hi);
	float4* s_lo = reinterpret_cast<float4*>(smem + L.lo);
	double* s_img = reinterpret_cast<double*>(smem + L.img);
	HalfPair* s_h16 = reinterpret_cast<HalfPair*>(smem + L.h16);
	__half* s_h = reinterpret_cast<__half*>(s_h16);
	int* s_cs = reinterpret_cast<int*>(smem + L.cstart);        // staged slot of each staged cell (65)
	unsigned short* s_list = reinterpret_cast<unsigned short*>(smem + L.lists);
	int* s_cnt = reinterpret_cast<int*>(smem + L.ccount);
	int* s_gst = reinterpret_cast<int*>(smem + L.gstart);
	double* s_ck = reinterpret_cast<double*>(smem + L.cell_k);
	double* s_csh = reinterpret_cast<double*>(smem + L.cell_shift);
	double* s_pd = reinterpret_cast<double*>(smem + L.params);  // eps24, sig2, shift6 (double)
	float* s_pf = reinterpret_cast<float*>(s_pd + 3 * KK);
	const Grid& g = bx.g;

	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int ns = p.ns;
	const int bxi = brick % bx.nb[0];
	const int byi = (brick / bx.nb[0]) % bx.nb[1];
	const int bzi = brick / (bx.nb[0] * bx.nb[1]);
	const int bc[3] = {bxi, byi, bzi};

	// staged cells k = lx + 4 ly + 16 lz, local l in 0..3, global 2b - 1 + l with periodic wrap
	if (tid < 64) {
		const int l[3] = {tid & 3, (tid >> 2) & 3, tid >> 4};
		int gc[3];
		for (int d = 0; d < 3; d++) {
			int gcd = 2 * bc[d] - 1 + l[d];
			double sh = 0.0;
			if (gcd < 0) {
				gcd += g.nc[d];
				sh = -g.L[d];
			} else if (gcd >= g.nc[d]) {
				gcd -= g.nc[d];
				sh = g.L[d];
			}
			gc[d] = gcd;
			s_csh[3 * tid + d] = sh;
			// frame: X = x + K, K = shift - c_brick + C
			const double cbr = (2 * bc[d] + 1) * g.cell_length[d];
			s_ck[3 * tid + d] = (sh - cbr) + (double) bx.frame_c[d];
		}
		const int gcell = bx.coff + (gc[2] * g.nc[1] + gc[1]) * g.nc[0] + gc[0];
		const int st = cstart[gcell];
		s_gst[tid] = st;
		s_cnt[tid] = max(0, cstart[gcell + 1] - st);
	}
	__syncthreads();
	// exclusive scan of the 64 staged-cell counts (warp 0, two per lane)
	if (warp == 0) {
		const int a = s_cnt[2 * lane], b = s_cnt[2 * lane + 1];
		int inc = a + b;
		for (int o = 1; o < 32; o <<= 1) {
			const int y = __shfl_up_sync(kFull, inc, o);
			if (lane >= o) inc += y;
		}
		const int excl = inc - (a + b);
		s_cs[2 * lane] = excl;
		s_cs[2 * lane + 1] = excl + a;
		if (lane == 31) s_cs[64] = inc;
	}
	__syncthreads();
	const int total = s_cs[64];
	const bool staged = total <= p.s_cap;

	// ---- staging: cell-major, each staged cell's molecules in their (id) order ---------------
	if (staged) {
		for (int c = warp; c < 64; c += kWarps) {
			const int st = s_gst[c], cnt = s_cnt[c], base = s_cs[c];
			const double kx = s_ck[3 * c], ky = s_ck[3 * c + 1], kz = s_ck[3 * c + 2];
			const double shx = s_csh[3 * c], shy = s_csh[3 * c + 1], shz = s_csh[3 * c + 2];
			for (int e = lane; e < cnt; e += 32) {
				const int gi = st + e;
				const double x = rx[gi], y = ry[gi], z = rz[gi];
				const double Xd = __dadd_rn(x, kx), Yd = __dadd_rn(y, ky), Zd = __dadd_rn(z, kz);
				const float X = __double2float_rn(Xd), Y = __double2float_rn(Yd), Z = __double2float_rn(Zd);
				const int slot_s = base + e;
				s_hi[slot_s] = make_float4(X, Y, Z, __int_as_float((gi << 3) | cid[gi]));
				// half-precision copy relative to the brick centre (slot pairs share one HalfPair)
				__half* hp = s_h + 8 * (slot_s >> 1) + (slot_s & 1);
				hp[0] = __float2half_rn(X - bx.frame_c[0]);
				hp[2] = __float2half_rn(Y - bx.frame_c[1]);
				hp[4] = __float2half_rn(Z - bx.frame_c[2]);
				if (kFP64) {
					s_img[slot_s] = __dadd_rn(x, shx);
					s_img[p.s_cap + slot_s] = __dadd_rn(y, shy);
					s_img[2 * p.s_cap + slot_s] = __dadd_rn(z, shz);
				} else {
					s_lo[slot_s] = make_float4(__double2float_rn(Xd - (double) X), __double2float_rn(Yd - (double) Y),
					                           __double2float_rn(Zd - (double) Z), 0.f);
				}
			}
		}
	}
	__syncthreads();

	// ---- pairs: warp w owns brick cell (1 + (w&1), 1 + ((w>>1)&1), 1 + (w>>2)) -----------------
	double U = 0.0, W = 0.0, NP = 0.0;
	bool same = false;
	const int il[3] = {1 + (warp & 1), 1 + ((warp >> 1) & 1), 1 + (warp >> 2)};
	const bool cell_ok = 2 * bxi + il[0] - 1 < g.nc[0] && 2 * byi + il[1] - 1 < g.nc[1] && 2 * bzi + il[2] - 1 < g.nc[2];
	const int icell = il[0] + 4 * il[1] + 16 * il[2];
	if (cell_ok && !staged) {
		// over capacity: gather from global memory
		const int st = s_gst[icell], cnt = s_cnt[icell];
		for (int e = lane; e < cnt; e += 32) {
			PairSums s = gather_pairs<!kFP64>(st + e, rx, ry, rz, cid, cstart, g, s_pd, ns, p.rc2, p.rclj2, bx.coff);
			fx[st + e] = s.F[0];
			fy[st + e] = s.F[1];
			fz[st + e] = s.F[2];
			U += s.U;
			W += s.W;
			NP += s.np;
			same |= s.same;
		}
	} else if (cell_ok) {
		const int i0 = s_cs[icell], ni = s_cs[icell + 1] - i0;
		unsigned short* mylist = s_list + warp * kCap * 32 + lane;
		for (int b0 = 0; b0 < ni; b0 += 32) {
			const bool act = b0 + lane < ni;
			const int slot_i = i0 + (act ? b0 + lane : 0);
			const float4 hi_i = s_hi[slot_i];
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
			int cnt = 0;
			double Fx = 0.0, Fy = 0.0, Fz = 0.0;
			const float eps24_1 = s_pf[0], sig2_1 = s_pf[KK], shift6_1 = s_pf[2 * KK];

			// one list entry in FP32 (branch-free: lanes past their list length or outside the
			// cutoff contribute zeros; the rare pairs within a few ulp of rc are decided in double)
			auto pair_fp32 = [&](int tt, float& ax, float& ay, float& az, float& au, float& aw, int& anp) {
				const bool v = tt < cnt;
				const int j = v ? (int) mylist[tt * 32] : slot_i;
				const float4 hj = s_hi[j];
				const float4 lj = s_lo[j];
				const float h0 = hi_i.x - hj.x, h1 = hi_i.y - hj.y, h2 = hi_i.z - hj.z;  // exact
				const float e0 = h0 + (lo_i.x - lj.x), e1 = h1 + (lo_i.y - lj.y), e2 = h2 + (lo_i.z - lj.z);
				const float d2f = fmaf(e0, e0, fmaf(e1, e1, e2 * e2));
				bool in = v && d2f < p.rc2f;
				const bool amb = v && fabsf(d2f - p.rc2f) <= p.band;
				if (__any_sync(kFull, amb)) {
					if (amb) {
						const double a0 = (double) h0 + ((double) lo_i.x - (double) lj.x);
						const double a1 = (double) h1 + ((double) lo_i.y - (double) lj.y);
						const double a2 = (double) h2 + ((double) lo_i.z - (double) lj.z);
						in = a0 * a0 + a1 * a1 + a2 * a2 < p.rc2;
					}
				}
				anp += in ? 1 : 0;
				same |= in && d2f == 0.f;
				const bool lj_in = kLjIsRc ? in : (in && d2f < p.rclj2f);
				float eps24, sig2, shift6;
				if (kSingle) {
					eps24 = eps24_1;
					sig2 = sig2_1;
					shift6 = shift6_1;
				} else {
					const int pk = ti * ns + (__float_as_int(hj.w) & 7);
					eps24 = s_pf[pk];
					sig2 = s_pf[KK + pk];
					shift6 = s_pf[2 * KK + pk];
				}
				const float inv = rcp_approx(lj_in ? d2f : 1.0f);
				const float s2 = sig2 * inv;
				const float s6 = s2 * s2 * s2;
				const float s12 = s6 * s6;
				const float m = s12 - s6;
				const float fac = lj_in ? eps24 * (s12 + m) * inv : 0.f;
				ax = fmaf(fac, e0, ax);
				ay = fmaf(fac, e1, ay);
				az = fmaf(fac, e2, az);
				au += lj_in ? fmaf(eps24, m, shift6) : 0.f;
				aw = fmaf(fac, d2f, aw);
			};
			auto pair_fp64 = [&](int tt, double& ax, double& ay, double& az, double& au, double& aw, int& anp) {
				if (tt >= cnt) return;
				const int j = mylist[tt * 32];
				const double d0 = __dsub_rn(xi, s_img[j]);
				const double d1 = __dsub_rn(yi, s_img[p.s_cap + j]);
				const double d2 = __dsub_rn(zi, s_img[2 * p.s_cap + j]);
				const double dd = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
				if (!(dd < p.rc2)) return;
				anp++;
				if (dd == 0.0) same = true;
				if (!(dd < p.rclj2)) return;
				int pk = 0;
				if (!kSingle) pk = ti * ns + (__float_as_int(s_hi[j].w) & 7);
				double f0, f1, f2, u, w;
				lj_pair_fp64(d0, d1, d2, dd, s_pd[pk], s_pd[KK + pk], s_pd[2 * KK + pk], f0, f1, f2, u, w);
				ax += f0;
				ay += f1;
				az += f2;
				au += u;
				aw = __dadd_rn(aw, w);
			};
			auto flush = [&]() {
				const int mx = __reduce_max_sync(kFull, cnt);
				int anp = 0;
				if (kFP64) {
					double ax[2] = {0, 0}, ay[2] = {0, 0}, az[2] = {0, 0}, au[2] = {0, 0}, aw[2] = {0, 0};
					for (int t = 0; t < mx; t += 2) {
#pragma unroll
						for (int u = 0; u < 2; u++) pair_fp64(t + u, ax[u], ay[u], az[u], au[u], aw[u], anp);
					}
					Fx += ax[0] + ax[1];
					Fy += ay[0] + ay[1];
					Fz += az[0] + az[1];
					U += au[0] + au[1];
					W = __dadd_rn(W, __dadd_rn(aw[0], aw[1]));
				} else {
					// four independent accumulator sets: four pair chains in flight per lane
					float ax[4] = {0.f, 0.f, 0.f, 0.f}, ay[4] = {0.f, 0.f, 0.f, 0.f}, az[4] = {0.f, 0.f, 0.f, 0.f};
					float au[4] = {0.f, 0.f, 0.f, 0.f}, aw[4] = {0.f, 0.f, 0.f, 0.f};
					for (int t = 0; t < mx; t += 4) {
#pragma unroll
						for (int u = 0; u < 4; u++) pair_fp32(t + u, ax[u], ay[u], az[u], au[u], aw[u], anp);
					}
					Fx += ((double) ax[0] + (double) ax[1]) + ((double) ax[2] + (double) ax[3]);
					Fy += ((double) ay[0] + (double) ay[1]) + ((double) ay[2] + (double) ay[3]);
					Fz += ((double) az[0] + (double) az[1]) + ((double) az[2] + (double) az[3]);
					U += ((double) au[0] + (double) au[1]) + ((double) au[2] + (double) au[3]);
					W += ((double) aw[0] + (double) aw[1]) + ((double) aw[2] + (double) aw[3]);
				}
				NP += (double) anp;
				cnt = 0;
			};

			// filter: the 9 rows of 3 staged cells around the i cell; every pair of consecutive
			// staged molecules is broadcast to all lanes and tested with packed half arithmetic
			const __half2 xi2 = __float2half2_rn(act ? hi_i.x - bx.frame_c[0] : 60000.f);
			const __half2 yi2 = __float2half2_rn(hi_i.y - bx.frame_c[1]);
			const __half2 zi2 = __float2half2_rn(hi_i.z - bx.frame_c[2]);
			const __half2 rc2h = __float2half2_rn(bx.rc2_h);
			// one 32-slot block [base, base + 32): per-lane hit mask, bit b = slot base + b
			auto block_mask = [&](int mb) -> unsigned {
				unsigned mask = 0u;
#pragma unroll
				for (int k = 0; k < 16; k++) {
					const HalfPair H = s_h16[mb + k];
					const __half2 dx = __hsub2(xi2, H.x), dy = __hsub2(yi2, H.y), dz = __hsub2(zi2, H.z);
					const __half2 d2 = __hfma2(dx, dx, __hfma2(dy, dy, __hmul2(dz, dz)));
					const unsigned hm = __hlt2_mask(d2, rc2h);
					mask |= ((hm & 1u) | ((hm >> 15) & 2u)) << (2 * k);
				}
				return mask;
			};
			for (int r = 0; r < 9; r++) {
				const int ky = il[1] + (r % 3) - 1, kz = il[2] + (r / 3) - 1;
				const int k0 = (il[0] - 1) + 4 * ky + 16 * kz;
				const int a = s_cs[k0], b = s_cs[k0 + 3];
				for (int base = a & ~1; base < b; base += 32) {
					unsigned mask = block_mask(base >> 1);
					// keep slots in [a, b) and drop i itself
					const int lo = a - base, hi = b - base;
					unsigned valid = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
					if (lo > 0) valid &= ~((1u << lo) - 1u);
					const int self = slot_i - base;
					if (self >= 0 && self < 32) valid &= ~(1u << self);
					mask &= valid;
					if (!act) mask = 0u;
					if (__reduce_max_sync(kFull, cnt + __popc(mask)) > kCap) flush();
					while (mask) {
						const int bit = __ffs(mask) - 1;
						mask &= mask - 1u;
						mylist[cnt * 32] = (unsigned short) (base + bit);
						cnt++;
					}
				}
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
	block_sum3_at(U, W, NP, partials, slot);
}

}  // namespace brick
}  // namespace mdgpu
