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
//           differences of their float "hi" parts are exact (Sterbenz), and the "lo" part X - hi
//           is kept as 9-bit fixed point (steps of 1/512 ulp of the binade) in the 4th word of the
//           same float4, with the component id: (hi_i - hi_j) + (lo_i - lo_j) is X_i - X_j to
//           about 2e-9 absolute, one 16-byte shared load per candidate. The FP64 mode also stages
//           the double image position x + shift.
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
	float lo_step[3];     // fixed-point step of the lo parts: 2^(k-32) for the binade [2^k, 2^(k+1))
	float lo_inv[3];      // 1 / lo_step
	float lo_c[3];        // -(2^23 + 256) * lo_step (decoding constant)
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

// list_cap: per-lane candidate list depth of the filter (0 for the list kernel, which reads its
// lists from global memory); half: whether the packed half-precision copy is staged.
__host__ __device__ inline SmemLayout layout(int s_cap, bool fp64, int list_cap, bool half = true) {
	SmemLayout L;
	size_t o = 0;
	L.hi = o;
	o = align16(o + sizeof(float4) * (s_cap + 1));   // + the far-away sentinel slot of the list kernel
	L.lo = o;
	L.img = o;
	if (fp64) o = align16(o + sizeof(double) * 3 * s_cap);
	L.h16 = o;
	if (half) o = align16(o + sizeof(HalfPair) * (s_cap / 2 + 20));  // 32-slot blocks may read past the end
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
inline int capacity_for(size_t budget, bool fp64, int list_cap, bool half = true) {
	int s_cap = 256;
	while (layout(s_cap + 64, fp64, list_cap, half).total <= budget) s_cap += 64;
	return s_cap > 65535 ? 65535 : s_cap;
}

// Frame constants of one box (host side).
// drift: how far a molecule may be outside its cell when staged (half the skin in the Verlet-skin
// mode, 0 otherwise).
inline void init_box(Box& b, const Grid& g, double rc, int32_t coff, double drift = 0.0) {
	b.g = g;
	b.coff = coff;
	for (int d = 0; d < 3; d++) {
		b.nb[d] = (g.nc[d] + 1) / 2;
		const double cl = g.cell_length[d];
		// smallest 2^k with the staged region X in [C - 2cl - drift, C + 2cl + drift] inside
		// [2^k, 2^(k+1)]
		double pk = 1.0;
		while (pk < 4.0 * cl + 2.0 * drift) pk *= 2.0;
		b.frame_c[d] = (float) (1.5 * pk);
		b.lo_step[d] = (float) std::ldexp(pk, -32);
		b.lo_inv[d] = (float) std::ldexp(1.0 / pk, 32);
		b.lo_c[d] = -8388864.0f * b.lo_step[d];
	}
	// half-precision filter: coordinates within +-2 cells of the brick centre; each rounding is at
	// most half an ulp of the largest coordinate, plus the rounding of the packed r^2 itself
	const double cmax = 2.0 * std::max(g.cell_length[0], std::max(g.cell_length[1], g.cell_length[2])) + drift;
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

// Views of the shared-memory layout.
struct Smem {
	float4* hi;
	double* img;
	HalfPair* h16;
	__half* h;
	int* cs;              // staged slot of each staged cell (65)
	unsigned short* list;
	int* cnt;
	int* gst;
	double* ck;
	double* csh;
	double* pd;           // eps24, sig2, shift6 (double)
	float* pf;            // the same as float
};

__device__ __forceinline__ Smem views(unsigned char* smem, const SmemLayout& L) {
	Smem S;
	S.hi = reinterpret_cast<float4*>(smem + L.hi);
	S.img = reinterpret_cast<double*>(smem + L.img);
	S.h16 = reinterpret_cast<HalfPair*>(smem + L.h16);
	S.h = reinterpret_cast<__half*>(S.h16);
	S.cs = reinterpret_cast<int*>(smem + L.cstart);
	S.list = reinterpret_cast<unsigned short*>(smem + L.lists);
	S.cnt = reinterpret_cast<int*>(smem + L.ccount);
	S.gst = reinterpret_cast<int*>(smem + L.gstart);
	S.ck = reinterpret_cast<double*>(smem + L.cell_k);
	S.csh = reinterpret_cast<double*>(smem + L.cell_shift);
	S.pd = reinterpret_cast<double*>(smem + L.params);
	S.pf = reinterpret_cast<float*>(S.pd + 3 * KK);
	return S;
}

// Warp w's brick cell: local (1 + (w&1), 1 + ((w>>1)&1), 1 + (w>>2)) in the 4x4x4 staged region;
// false when it lies beyond the grid (odd cell counts: the last brick of a dimension is partial).
__device__ __forceinline__ bool own_cell(const Box& bx, int brick, int w, int& icell) {
	const int bxi = brick % bx.nb[0];
	const int byi = (brick / bx.nb[0]) % bx.nb[1];
	const int bzi = brick / (bx.nb[0] * bx.nb[1]);
	const int il[3] = {1 + (w & 1), 1 + ((w >> 1) & 1), 1 + (w >> 2)};
	icell = il[0] + 4 * il[1] + 16 * il[2];
	return 2 * bxi + il[0] - 1 < bx.g.nc[0] && 2 * byi + il[1] - 1 < bx.g.nc[1] && 2 * bzi + il[2] - 1 < bx.g.nc[2];
}

// The packed 4th word of a staged molecule: lo parts as 9-bit fields (value + 256, bits 0-8, 9-17,
// 18-26) in steps of Box::lo_step, component id in bits 27-29.
__device__ __forceinline__ unsigned pack_lo(float lx, float ly, float lz, int cid, const Box& bx) {
	const float l[3] = {lx, ly, lz};
	unsigned w = (unsigned) cid << 27;
	for (int d = 0; d < 3; d++) {
		int q = __float2int_rn(l[d] * bx.lo_inv[d]);   // power-of-two step: exact product
		q = max(-255, min(255, q));
		w |= (unsigned) (q + 256) << (9 * d);
	}
	return w;
}

// lo = fma(2^23 + field, step, -(2^23 + 256) * step): exact in one FMA (power-of-two step).
__device__ __forceinline__ float3 unpack_lo(unsigned w, const Box& bx) {
	return make_float3(fmaf(__uint_as_float(0x4B000000u | (w & 511u)), bx.lo_step[0], bx.lo_c[0]),
	                   fmaf(__uint_as_float(0x4B000000u | ((w >> 9) & 511u)), bx.lo_step[1], bx.lo_c[1]),
	                   fmaf(__uint_as_float(0x4B000000u | ((w >> 18) & 511u)), bx.lo_step[2], bx.lo_c[2]));
}

__device__ __forceinline__ int unpack_cid(unsigned w) { return (int) ((w >> 27) & 7u); }

// Stages molecule e of staged cell c at double position (x, y, z), component q: the hi/lo frame
// position, and the half-precision copy or the double image as the staging mode asks.
// The same with the cell's frame offset (kx, ky, kz) and image shift (shx, shy, shz) given, at slot
// slot_s.
template <bool kFP64, bool kHalf>
__device__ __forceinline__ void stage_at(const Const& p, const Box& bx, const Smem& S, int slot_s, double x, double y,
                                         double z, int q, double kx, double ky, double kz, double shx, double shy,
                                         double shz) {
	const double Xd = __dadd_rn(x, kx), Yd = __dadd_rn(y, ky), Zd = __dadd_rn(z, kz);
	const float X = __double2float_rn(Xd), Y = __double2float_rn(Yd), Z = __double2float_rn(Zd);
	const unsigned w = pack_lo(__double2float_rn(Xd - (double) X), __double2float_rn(Yd - (double) Y),
	                           __double2float_rn(Zd - (double) Z), q, bx);
	S.hi[slot_s] = make_float4(X, Y, Z, __uint_as_float(w));
	if (kHalf) {
		// half-precision copy relative to the brick centre (slot pairs share one HalfPair)
		__half* hp = S.h + 8 * (slot_s >> 1) + (slot_s & 1);
		hp[0] = __float2half_rn(X - bx.frame_c[0]);
		hp[2] = __float2half_rn(Y - bx.frame_c[1]);
		hp[4] = __float2half_rn(Z - bx.frame_c[2]);
	}
	if (kFP64) {
		S.img[slot_s] = __dadd_rn(x, shx);
		S.img[p.s_cap + slot_s] = __dadd_rn(y, shy);
		S.img[2 * p.s_cap + slot_s] = __dadd_rn(z, shz);
	}
}

template <bool kFP64, bool kHalf>
__device__ __forceinline__ void stage_one(const Const& p, const Box& bx, const Smem& S, int c, int e, double x,
                                          double y, double z, int q) {
	stage_at<kFP64, kHalf>(p, bx, S, S.cs[c] + e, x, y, z, q, S.ck[3 * c], S.ck[3 * c + 1], S.ck[3 * c + 2],
	                       S.csh[3 * c], S.csh[3 * c + 1], S.csh[3 * c + 2]);
}

// Stages the 4x4x4 cells around brick `brick` (positions in the local frame; double images in the
// FP64 mode). Returns false when the region exceeds the staged capacity (nothing staged then; the
// cell ranges s_gst/s_cnt are set either way). Ends with a CTA barrier.
template <bool kFP64, bool kHalf = true, bool kWide = true>
__device__ __forceinline__ bool stage(const Const& p, const Box& bx, int brick, const Smem& S, const double* rx,
                                      const double* ry, const double* rz, const int32_t* cid, const int32_t* cstart) {
	const Grid& g = bx.g;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int bc[3] = {brick % bx.nb[0], (brick / bx.nb[0]) % bx.nb[1], brick / (bx.nb[0] * bx.nb[1])};
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
			S.csh[3 * tid + d] = sh;
			// frame: X = x + K, K = shift - c_brick + C
			const double cbr = (2 * bc[d] + 1) * g.cell_length[d];
			S.ck[3 * tid + d] = (sh - cbr) + (double) bx.frame_c[d];
		}
		const int gcell = bx.coff + (gc[2] * g.nc[1] + gc[1]) * g.nc[0] + gc[0];
		const int st = cstart[gcell];
		S.gst[tid] = st;
		S.cnt[tid] = max(0, cstart[gcell + 1] - st);
	}
	__syncthreads();
	// exclusive scan of the 64 staged-cell counts (warp 0, two per lane)
	if (warp == 0) {
		const int a = S.cnt[2 * lane], b = S.cnt[2 * lane + 1];
		int inc = a + b;
		for (int o = 1; o < 32; o <<= 1) {
			const int y = __shfl_up_sync(kFull, inc, o);
			if (lane >= o) inc += y;
		}
		const int excl = inc - (a + b);
		S.cs[2 * lane] = excl;
		S.cs[2 * lane + 1] = excl + a;
		if (lane == 31) S.cs[64] = inc;
	}
	__syncthreads();
	const bool staged = S.cs[64] <= p.s_cap;
	// cell-major, each staged cell's molecules in their (id) order. A warp stages cells warp,
	// warp + 8, ...; kWide: four cells per round, every load of the round issued before the first
	// store (the stores to shared memory would otherwise hold back the next cell's loads). The
	// persistent ensemble kernel, at its register limit, stages one cell at a time.
	if (staged && !kWide) {
		for (int c = warp; c < 64; c += kWarps) {
			const int st = S.gst[c], cnt = S.cnt[c], base = S.cs[c];
			const double kx = S.ck[3 * c], ky = S.ck[3 * c + 1], kz = S.ck[3 * c + 2];
			const double shx = S.csh[3 * c], shy = S.csh[3 * c + 1], shz = S.csh[3 * c + 2];
			for (int e = lane; e < cnt; e += 32) {
				const int gi = st + e;
				stage_at<kFP64, kHalf>(p, bx, S, base + e, rx[gi], ry[gi], rz[gi], cid[gi], kx, ky, kz, shx, shy, shz);
			}
		}
	}
	if (staged && kWide) {
		for (int c0 = warp; c0 < 64; c0 += 4 * kWarps) {
			double x[4], y[4], z[4];
			int q[4];
#pragma unroll
			for (int u = 0; u < 4; u++) {
				const int c = c0 + u * kWarps;
				const int gi = S.gst[c] + lane;
				const bool a = lane < S.cnt[c];
				x[u] = a ? rx[gi] : 0.0;
				y[u] = a ? ry[gi] : 0.0;
				z[u] = a ? rz[gi] : 0.0;
				q[u] = a ? cid[gi] : 0;
			}
#pragma unroll
			for (int u = 0; u < 4; u++) {
				const int c = c0 + u * kWarps;
				const int cnt = S.cnt[c];
				if (lane < cnt) stage_one<kFP64, kHalf>(p, bx, S, c, lane, x[u], y[u], z[u], q[u]);
				for (int e = lane + 32; e < cnt; e += 32) {
					const int gi = S.gst[c] + e;
					stage_one<kFP64, kHalf>(p, bx, S, c, e, rx[gi], ry[gi], rz[gi], cid[gi]);
				}
			}
		}
	}
	__syncthreads();
	return staged;
}

// Cutoff decision for a pair within a few ulp of rc (rare): recomputed from the FP64 positions in
// global memory with the FP64 path's operations (xi - (x_j + shift), sum of squares), so that the
// mixed mode evaluates exactly the pairs the FP64 mode evaluates. j is a staged slot; its cell is
// found by bisection of the staged-cell starts.
static __device__ __noinline__ bool exact_cut(const Smem& S, double rc2, int j, int gi, const double* rx, const double* ry,
                                       const double* rz) {
	int lo = 0, hi = 63;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (S.cs[mid] <= j)
			lo = mid;
		else
			hi = mid - 1;
	}
	const int gj = S.gst[lo] + (j - S.cs[lo]);
	const double d0 = __dsub_rn(rx[gi], __dadd_rn(rx[gj], S.csh[3 * lo]));
	const double d1 = __dsub_rn(ry[gi], __dadd_rn(ry[gj], S.csh[3 * lo + 1]));
	const double d2 = __dsub_rn(rz[gi], __dadd_rn(rz[gj], S.csh[3 * lo + 2]));
	const double dd = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
	return dd < rc2;
}

// One list entry j of molecule i in FP32 with FP64-ready accumulators (branch-free: an invalid
// entry, v = false, or a pair outside the cutoff contributes zeros; the rare pairs within a few ulp
// of rc are decided in double from the same hi/lo parts).
template <bool kSingle, bool kLjIsRc>
__device__ __forceinline__ void lj32(const Const& p, bool v, const float4& hi_i, const float3& lo_i, int ti, int ns,
                                     const float4 hj, const Box& bx, const float* pf, float eps24_1, float sig2_1,
                                     float shift6_1, float& ax, float& ay, float& az, float& au, float& aw, int& anp,
                                     bool& same, const Smem& S, int j, int gi, const double* rx, const double* ry,
                                     const double* rz) {
	const float3 lj = unpack_lo(__float_as_uint(hj.w), bx);
	const float h0 = hi_i.x - hj.x, h1 = hi_i.y - hj.y, h2 = hi_i.z - hj.z;  // exact
	const float e0 = h0 + (lo_i.x - lj.x), e1 = h1 + (lo_i.y - lj.y), e2 = h2 + (lo_i.z - lj.z);
	const float d2f = fmaf(e0, e0, fmaf(e1, e1, e2 * e2));
	bool in = v && d2f < p.rc2f;
	const bool amb = v && fabsf(d2f - p.rc2f) <= p.band;
	if (amb) in = exact_cut(S, p.rc2, j, gi, rx, ry, rz);
	anp += in ? 1 : 0;
	same |= in && d2f == 0.f;
	const bool lj_in = kLjIsRc ? in : (in && d2f < p.rclj2f);
	float eps24, sig2, shift6;
	if (kSingle) {
		eps24 = eps24_1;
		sig2 = sig2_1;
		shift6 = shift6_1;
	} else {
		const int pk = ti * ns + unpack_cid(__float_as_uint(hj.w));
		eps24 = pf[pk];
		sig2 = pf[KK + pk];
		shift6 = pf[2 * KK + pk];
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
}

// One list entry j (staged slot) of molecule i at the double image position (xi, yi, zi), in FP64
// with the reference's operation order.
template <bool kSingle>
__device__ __forceinline__ void lj64(const Const& p, double xi, double yi, double zi, int ti, int ns, int j,
                                     const Smem& S, double& ax, double& ay, double& az, double& au, double& aw,
                                     int& anp, bool& same) {
	const double d0 = __dsub_rn(xi, S.img[j]);
	const double d1 = __dsub_rn(yi, S.img[p.s_cap + j]);
	const double d2 = __dsub_rn(zi, S.img[2 * p.s_cap + j]);
	const double dd = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
	if (!(dd < p.rc2)) return;
	anp++;
	if (dd == 0.0) same = true;
	if (!(dd < p.rclj2)) return;
	int pk = 0;
	if (!kSingle) pk = ti * ns + unpack_cid(__float_as_uint(S.hi[j].w));
	double f0, f1, f2, u, w;
	lj_pair_fp64(d0, d1, d2, dd, S.pd[pk], S.pd[KK + pk], S.pd[2 * KK + pk], f0, f1, f2, u, w);
	ax += f0;
	ay += f1;
	az += f2;
	au += u;
	aw = __dadd_rn(aw, w);
}

// Neighbour lists of the Verlet-skin mode: entry k of molecule i (sorted slot) is a staged slot of
// i's brick region, stored at ((k/8)*n + i)*8 + k%8, so that one 16-byte load gives a lane 8 entries
// and a warp's loads are contiguous; count[i] entries, kListOverflow when more than cap were found.
struct Lists {
	unsigned short* nbr;
	unsigned short* count;
	double *rx_ref, *ry_ref, *rz_ref;   // positions at the build
	int64_t n;
	int cap;
	unsigned long long* builds;        // incremented once per build
	int sentinel;                      // staged slot of the list kernel's far-away sentinel
	unsigned char* kind;               // per brick: 1 = sparse (evaluated one warp per brick)
	unsigned* counts;                  // sparse [0] and dense [1] bricks of the build (or null)
	int32_t* blist;                    // dense bricks at [0, nbricks), sparse ones from nbricks on
	int nbricks;
	PruneState* pst;                   // pruned lists: their state (the evaluation's last CTA updates it)
	int step;                          // id of the step being evaluated
};
// A brick is sparse when its whole staged region holds at most kSparseCap molecules and its own
// cells at most 32: one warp stages and evaluates it, without CTA-wide barriers.
constexpr int kSparseCap = 128;
constexpr unsigned short kListOverflow = 0xffff;

// Forces on the molecules of brick `brick` (index within its box) of box `bx`; U, W and the pair
// count go to partials[slot]. The pair table must already be in shared memory (load_params).
// Ends with a CTA-wide barrier after which no thread reads the staged data.
template <bool kFP64, bool kSingle, bool kLjIsRc, int kCap, bool kWide = true>
__device__ __forceinline__ void pairs(const Const& p, const Box& bx, int brick, int64_t slot, unsigned char* smem,
                                      const double* rx, const double* ry, const double* rz, const int32_t* cid,
                                      const int32_t* cstart, double* fx, double* fy, double* fz, double* partials,
                                      int* status) {
	const SmemLayout L = layout(p.s_cap, kFP64, kCap);
	const Smem S = views(smem, L);
	float4* s_hi = S.hi;
	double* s_img = S.img;
	HalfPair* s_h16 = S.h16;
	int* s_cs = S.cs;
	unsigned short* s_list = S.list;
	int* s_cnt = S.cnt;
	int* s_gst = S.gst;
	double* s_pd = S.pd;
	float* s_pf = S.pf;
	const Grid& g = bx.g;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int ns = p.ns;
	const bool staged = stage<kFP64, true, kWide>(p, bx, brick, S, rx, ry, rz, cid, cstart);

	// ---- pairs: warp w owns brick cell (1 + (w&1), 1 + ((w>>1)&1), 1 + (w>>2)) -----------------
	double U = 0.0, W = 0.0, NP = 0.0;
	bool same = false;
	const int il[3] = {1 + (warp & 1), 1 + ((warp >> 1) & 1), 1 + (warp >> 2)};
	int icell;
	const bool cell_ok = own_cell(bx, brick, warp, icell);
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
			const float3 lo_i = unpack_lo(__float_as_uint(hi_i.w), bx);
			double xi = 0, yi = 0, zi = 0;
			if (kFP64) {
				xi = s_img[slot_i];
				yi = s_img[p.s_cap + slot_i];
				zi = s_img[2 * p.s_cap + slot_i];
			}
			const int ti = unpack_cid(__float_as_uint(hi_i.w));
			const int gi = s_gst[icell] + (slot_i - i0);
			int cnt = 0;
			double Fx = 0.0, Fy = 0.0, Fz = 0.0;
			const float eps24_1 = s_pf[0], sig2_1 = s_pf[KK], shift6_1 = s_pf[2 * KK];

			// one list entry in FP32 (branch-free: lanes past their list length or outside the
			// cutoff contribute zeros; the rare pairs within a few ulp of rc are decided in double)
			auto pair_fp32 = [&](int tt, float& ax, float& ay, float& az, float& au, float& aw, int& anp) {
				const bool v = tt < cnt;
				const int j = v ? (int) mylist[tt * 32] : slot_i;
				lj32<kSingle, kLjIsRc>(p, v, hi_i, lo_i, ti, ns, s_hi[j], bx, s_pf, eps24_1, sig2_1, shift6_1, ax, ay, az,
				                       au, aw, anp, same, S, j, gi, rx, ry, rz);
			};
			auto pair_fp64 = [&](int tt, double& ax, double& ay, double& az, double& au, double& aw, int& anp) {
				if (tt >= cnt) return;
				lj64<kSingle>(p, xi, yi, zi, ti, ns, mylist[tt * 32], S, ax, ay, az, au, aw, anp, same);
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

// Entries of each lane's write-combining ring in build_lists: up to 7 unwritten entries plus the
// 32 that one block of candidates can add; a power of two for the index wrap.
constexpr int kBuildRing = 64;

// Shared-memory bytes of build_lists for a staged capacity s_cap.
__host__ __device__ inline size_t build_bytes(int s_cap) {
	return align16(sizeof(HalfPair) * (s_cap / 2 + 20)) + align16(sizeof(int) * 65) + 2 * align16(sizeof(int) * 64) +
	       align16(sizeof(double) * 3 * 64) + sizeof(unsigned short) * kBuildRing * kThreads;
}

// Bits [lo, hi) of a 16-bit field (0 <= lo, hi <= 16).
__device__ __forceinline__ unsigned range16(int lo, int hi) {
	const unsigned up = hi >= 16 ? 0xffffu : ((1u << hi) - 1u);
	return lo >= 16 ? 0u : up & ~((1u << lo) - 1u);
}

// Verlet-skin build for brick `brick`: stages the half-precision copy of the 4x4x4 cells around it
// (the same slots as stage() gives them) and writes to each own molecule's list every candidate
// that the packed filter finds within the list radius (bx.rc2_h holds rc + skin plus the rounding
// margin), with the positions of the build. No forces: list_pairs evaluates the lists.
__device__ __forceinline__ void build_lists(const Box& bx, int brick, int s_cap, unsigned char* smem,
                                            const double* rx, const double* ry, const double* rz,
                                            const int32_t* cstart, Lists lists, int64_t kind_slot) {
	HalfPair* s_h16 = reinterpret_cast<HalfPair*>(smem);
	__half* s_h = reinterpret_cast<__half*>(smem);
	size_t o = align16(sizeof(HalfPair) * (s_cap / 2 + 20));
	int* s_cs = reinterpret_cast<int*>(smem + o);
	o += align16(sizeof(int) * 65);
	int* s_cnt = reinterpret_cast<int*>(smem + o);
	o += align16(sizeof(int) * 64);
	int* s_gst = reinterpret_cast<int*>(smem + o);
	o += align16(sizeof(int) * 64);
	double* s_ck = reinterpret_cast<double*>(smem + o);
	o += align16(sizeof(double) * 3 * 64);
	const Grid& g = bx.g;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	unsigned short* ring = reinterpret_cast<unsigned short*>(smem + o) + kBuildRing * tid;
	const int bc[3] = {brick % bx.nb[0], (brick / bx.nb[0]) % bx.nb[1], brick / (bx.nb[0] * bx.nb[1])};
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
			const double cbr = (2 * bc[d] + 1) * g.cell_length[d];
			s_ck[3 * tid + d] = (sh - cbr) + (double) bx.frame_c[d];
		}
		const int gcell = bx.coff + (gc[2] * g.nc[1] + gc[1]) * g.nc[0] + gc[0];
		const int st = cstart[gcell];
		s_gst[tid] = st;
		s_cnt[tid] = max(0, cstart[gcell + 1] - st);
	}
	__syncthreads();
	if (warp == 0) {
		const int a = s_cnt[2 * lane], b = s_cnt[2 * lane + 1];
		int inc = a + b;
		for (int of = 1; of < 32; of <<= 1) {
			const int y = __shfl_up_sync(kFull, inc, of);
			if (lane >= of) inc += y;
		}
		const int excl = inc - (a + b);
		s_cs[2 * lane] = excl;
		s_cs[2 * lane + 1] = excl + a;
		if (lane == 31) s_cs[64] = inc;
	}
	__syncthreads();
	const bool staged = s_cs[64] <= s_cap;
	if (staged) {
		for (int c = warp; c < 64; c += kWarps) {
			const int st = s_gst[c], cnt = s_cnt[c], base = s_cs[c];
			const double kx = s_ck[3 * c], ky = s_ck[3 * c + 1], kz = s_ck[3 * c + 2];
			for (int e = lane; e < cnt; e += 32) {
				const int gi = st + e;
				const float X = __double2float_rn(__dadd_rn(rx[gi], kx));
				const float Y = __double2float_rn(__dadd_rn(ry[gi], ky));
				const float Z = __double2float_rn(__dadd_rn(rz[gi], kz));
				const int slot_s = base + e;
				__half* hp = s_h + 8 * (slot_s >> 1) + (slot_s & 1);
				hp[0] = __float2half_rn(X - bx.frame_c[0]);
				hp[2] = __float2half_rn(Y - bx.frame_c[1]);
				hp[4] = __float2half_rn(Z - bx.frame_c[2]);
			}
		}
	}
	__syncthreads();
	int icell;
	if (own_cell(bx, brick, warp, icell)) {
		const int st = s_gst[icell], ncell = s_cnt[icell], i0 = s_cs[icell];
		const int il[3] = {1 + (warp & 1), 1 + ((warp >> 1) & 1), 1 + (warp >> 2)};
		if (!staged) {
			for (int e = lane; e < ncell; e += 32) {
				lists.count[st + e] = kListOverflow;
				lists.rx_ref[st + e] = rx[st + e];
				lists.ry_ref[st + e] = ry[st + e];
				lists.rz_ref[st + e] = rz[st + e];
			}
		} else {
			const __half2 rc2h = __float2half2_rn(bx.rc2_h);
			// each lane's entries go through its ring in shared memory and leave it in blocks of
			// 8 (one 16-byte store each); the rotation by lane spreads the ring writes over banks
			const int rot = 8 * (lane & 7);
			for (int b0 = 0; b0 < ncell; b0 += 32) {
				const bool act = b0 + lane < ncell;
				const int slot_i = i0 + (act ? b0 + lane : 0);
				const int gi = st + (slot_i - i0);
				const __half* hi = s_h + 8 * (slot_i >> 1) + (slot_i & 1);
				const __half2 xi2 = act ? __half2half2(hi[0]) : __float2half2_rn(60000.f);
				const __half2 yi2 = __half2half2(hi[2]);
				const __half2 zi2 = __half2half2(hi[4]);
				uint4* dst = reinterpret_cast<uint4*>(lists.nbr) + gi;
				int cnt = 0, done = 0;   // entries found; entries written (a multiple of 8)
				for (int r = 0; r < 9; r++) {
					const int ky = il[1] + (r % 3) - 1, kz = il[2] + (r / 3) - 1;
					const int k0 = (il[0] - 1) + 4 * ky + 16 * kz;
					const int a = s_cs[k0], b = s_cs[k0 + 3];
					for (int base = a & ~1; base < b; base += 32) {
						// bit k: slot base + 2k, bit 16 + k: slot base + 2k + 1
						unsigned mask = 0u;
#pragma unroll
						for (int k = 0; k < 16; k++) {
							const HalfPair H = s_h16[(base >> 1) + k];
							const __half2 dx = __hsub2(xi2, H.x), dy = __hsub2(yi2, H.y), dz = __hsub2(zi2, H.z);
							const __half2 d2 = __hfma2(dx, dx, __hfma2(dy, dy, __hmul2(dz, dz)));
							mask |= __hlt2_mask(d2, rc2h) & ((1u << k) | (1u << (16 + k)));
						}
						// keep slots in [a, b) and drop i itself
						const int lo = a - base, hi_b = b - base;
						mask &= range16(max(0, (lo + 1) >> 1), min(16, (hi_b + 1) >> 1)) |
						        (range16(max(0, lo >> 1), min(16, hi_b >> 1)) << 16);
						const int self = slot_i - base;
						if (self >= 0 && self < 32) mask &= ~(1u << ((self & 1) * 16 + (self >> 1)));
						if (!act) mask = 0u;
						while (mask) {
							const int bit = __ffs(mask) - 1;
							mask &= mask - 1u;
							ring[(cnt + rot) & (kBuildRing - 1)] = (unsigned short) (base + 2 * (bit & 15) + (bit >> 4));
							cnt++;
						}
						for (; done + 8 <= cnt; done += 8)
							if (done < lists.cap)
								dst[(int64_t) (done >> 3) * lists.n] =
								    *reinterpret_cast<const uint4*>(ring + ((done + rot) & (kBuildRing - 1)));
					}
				}
				if (act) {
					// the last block of 8, padded with the list kernel's sentinel slot
					if (cnt > done) {
						for (int k = cnt; k < done + 8; k++)
							ring[(k + rot) & (kBuildRing - 1)] = (unsigned short) lists.sentinel;
						if (done < lists.cap)
							dst[(int64_t) (done >> 3) * lists.n] =
							    *reinterpret_cast<const uint4*>(ring + ((done + rot) & (kBuildRing - 1)));
					}
					lists.count[gi] = cnt <= lists.cap ? (unsigned short) cnt : kListOverflow;
					lists.rx_ref[gi] = rx[gi];
					lists.ry_ref[gi] = ry[gi];
					lists.rz_ref[gi] = rz[gi];
				}
			}
		}
	}
	if (tid == 0) {
		int n_own = 0;
		for (int w = 0; w < kWarps; w++) {
			int ic;
			if (own_cell(bx, brick, w, ic)) n_own += s_cnt[ic];
		}
		const bool sparse = s_cs[64] <= kSparseCap && n_own <= 32;
		lists.kind[kind_slot] = sparse ? 1 : 0;
		if (lists.counts) {
			const unsigned at = atomicAdd(lists.counts + (sparse ? 0 : 1), 1u);
			lists.blist[(sparse ? lists.nbricks : 0) + (int) at] = (int32_t) kind_slot;
		}
		if (brick == 0) atomicAdd(lists.builds, 1ull);
	}
}

// What the list kernels do with a molecule's force once it is summed. Mode 0 stores it. Modes 1
// and 2 apply the closing kick of the step, v += (dt/2m) F, and add m v^2 to the step's sum
// (Molecule::upd_postF, molecules/Molecule.cpp:193-205); mode 2 (the last step of a run) stores F
// and v, mode 1 goes on with the opening kick and drift of the next step, v = 1*v + (dt/2m) F,
// r' = r + dt v (Molecule::upd_preF with vcorr = 1, Molecule.cpp:128-135), writes r' to the other
// position buffer (other bricks still stage r) and flags a rebuild with `id` when r' is farther than
// skin/2 from the position of the last build. Same operations and roundings as the Leapfrog kernels.
// The CTA's largest squared drift of a list kernel with pruned lists (float bits; set to 0 before the
// first finish, flushed by drift_flush).
__device__ __forceinline__ unsigned& drift_slot() {
	__shared__ unsigned s_drift;
	return s_drift;
}

struct Kick {
	int mode;
	int id;
	double dt;
	double half2;                 // (skin/2)^2
	double post[kMaxSpecies];     // (0.5 dt) / m of the closing kick
	double pre[kMaxSpecies];      // (0.5 dt) / m of the opening kick
	double mass[kMaxSpecies];
	double *vx, *vy, *vz;
	double *ox, *oy, *oz;         // positions after the drift (mode 1)
	int* flag;
	unsigned* dmax;               // mode 1 with pruned lists: the largest squared drift, as float bits
};

__device__ __forceinline__ double finish(const Kick& k, int64_t gi, double Fx, double Fy, double Fz, const double* rx,
                                         const double* ry, const double* rz, const int32_t* cid, const Lists& lists,
                                         double* fx, double* fy, double* fz, int* status) {
	if (!(Fx == Fx && Fy == Fy && Fz == Fz) || isinf(Fx) || isinf(Fy) || isinf(Fz)) atomicOr(status, kStatusNonFinite);
	if (k.mode != 1) {
		fx[gi] = Fx;
		fy[gi] = Fy;
		fz[gi] = Fz;
	}
	if (k.mode == 0) return 0.0;
	const int t = cid[gi];
	const double a = k.post[t];
	const double vx = __dadd_rn(k.vx[gi], __dmul_rn(a, Fx));
	const double vy = __dadd_rn(k.vy[gi], __dmul_rn(a, Fy));
	const double vz = __dadd_rn(k.vz[gi], __dmul_rn(a, Fz));
	const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
	if (!(v2 == v2) || isinf(v2)) atomicOr(status, kStatusNonFinite);
	const double mv2 = __dmul_rn(k.mass[t], v2);
	if (k.mode == 2) {
		k.vx[gi] = vx;
		k.vy[gi] = vy;
		k.vz[gi] = vz;
		return mv2;
	}
	const double b = k.pre[t];
	const double wx = __dadd_rn(__dmul_rn(1.0, vx), __dmul_rn(b, Fx));
	const double wy = __dadd_rn(__dmul_rn(1.0, vy), __dmul_rn(b, Fy));
	const double wz = __dadd_rn(__dmul_rn(1.0, vz), __dmul_rn(b, Fz));
	const double x0 = rx[gi], y0 = ry[gi], z0 = rz[gi];
	const double x = __dadd_rn(x0, __dmul_rn(k.dt, wx));
	const double y = __dadd_rn(y0, __dmul_rn(k.dt, wy));
	const double z = __dadd_rn(z0, __dmul_rn(k.dt, wz));
	if (k.dmax) {
		// this drift's length squared, rounded up (the bits of a non-negative float order as it does)
		const double sx = x - x0, sy = y - y0, sz = z - z0;
		atomicMax(&drift_slot(), __float_as_uint(__double2float_ru(sx * sx + sy * sy + sz * sz)));
	}
	k.vx[gi] = wx;
	k.vy[gi] = wy;
	k.vz[gi] = wz;
	k.ox[gi] = x;
	k.oy[gi] = y;
	k.oz[gi] = z;
	const double dx = x - lists.rx_ref[gi], dy = y - lists.ry_ref[gi], dz = z - lists.rz_ref[gi];
	if (!(dx * dx + dy * dy + dz * dz <= k.half2)) *k.flag = k.id;
	return mv2;
}

// The CTA's largest squared drift into *dmax (thread 0, after a CTA barrier that follows every
// finish; the atomic is skipped when the value there is already as large).
__device__ __forceinline__ void drift_flush(unsigned* dmax) {
	if (dmax && threadIdx.x == 0 && drift_slot() > __ldcg(dmax)) atomicMax(dmax, drift_slot());
}

// Lanes per molecule for g molecules on one warp: the largest power of two with lpm * g <= 32.
__device__ __forceinline__ int lanes_per_molecule(int g) {
	int lpm = 1;
	while (lpm * 2 * g <= 32) lpm *= 2;
	return lpm;
}

#ifndef MDGPU_LIST_ACC
#define MDGPU_LIST_ACC 1
#endif
// Independent FP32 partial sums per lane in list_chunk (entry u of a block of 8 goes to u % kListAcc).
constexpr int kListAcc = MDGPU_LIST_ACC;
static_assert(kListAcc == 1 || kListAcc == 2 || kListAcc == 4, "1, 2 or 4 partial sums");

// Word k of a block of 8 list entries (register selection; k need not be a constant).
__device__ __forceinline__ unsigned list_word(const uint4& v, int k) {
	return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w;
}

// The partial sums in a fixed order, in FP64.
__device__ __forceinline__ double acc_sum(const float* a) {
	if (kListAcc == 4) return ((double) a[0] + (double) a[1]) + ((double) a[2] + (double) a[3]);
	if (kListAcc == 2) return (double) a[0] + (double) a[1 % kListAcc];
	return (double) a[0];
}

// Where the evaluation of a prune step writes the inner lists: the entries of each molecule's build
// list whose squared staged distance is below rp2f, in list order, in the layout of Lists::nbr.
struct PruneOut {
	unsigned short* nbr;
	unsigned short* count;
	float rp2f;
};

// Entries of each thread's ring in shared memory in a prune step: up to 7 unwritten entries plus the
// 8 of one block; entry k of thread t at k * kThreads + t (a warp's stores of one entry each fall in
// 16 banks). The prune variant's shared memory is the layout's plus kPruneRingBytes.
constexpr int kPruneRing = 16;
constexpr size_t kPruneRingBytes = sizeof(unsigned short) * kPruneRing * kThreads;

// A warp evaluates the lists of the brick's own molecules t0 .. t1-1 (in the order of the own cells
// own[0..8] / ocell[0..7]), lpm lanes per molecule (a power of two, (t1 - t0) * lpm <= 32): lane
// sub = lane % lpm takes the blocks sub, sub + lpm, ... of its molecule's list, the lanes' forces
// are summed by a fixed butterfly and the molecule is finished by its first lane; U, W, the pair
// count and the same-position flag are accumulated into the caller's sums. kPrune (a prune step): the
// entries also pass the prune test into the molecule's inner list (po).
template <bool kFP64, bool kSingle, bool kLjIsRc, bool kClampJ = false, bool kPrune = false>
__device__ __forceinline__ void list_chunk(const Const& p, const Box& bx, const Smem& S, const int* s_own,
                                           const int* s_ocell, int t0, int t1, int lpm, const double* rx,
                                           const double* ry,
                                           const double* rz, const int32_t* cid, const int32_t* cstart, double* fx,
                                           double* fy, double* fz, int* status, const Lists& lists, const Kick& kick,
                                           double& U, double& W, double& NP, double& MV, bool& same,
                                           const PruneOut& po = PruneOut{}, unsigned short* ring = nullptr) {
	const int lane = threadIdx.x & 31;
	const int ns = p.ns;
	const float eps24_1 = S.pf[0], sig2_1 = S.pf[KK], shift6_1 = S.pf[2 * KK];
	const int sub = lane & (lpm - 1);
	const int t = t0 + lane / lpm;
	const bool act = t < t1;
	int w = 0;
	if (act)
		while (w < 7 && s_own[w + 1] <= t) w++;
	const int slot_i = act ? S.cs[s_ocell[w]] + (t - s_own[w]) : 0;
	const float4 hi_i = S.hi[slot_i];
	const float3 lo_i = unpack_lo(__float_as_uint(hi_i.w), bx);
	double xi = 0, yi = 0, zi = 0;
	if (kFP64) {
		xi = S.img[slot_i];
		yi = S.img[p.s_cap + slot_i];
		zi = S.img[2 * p.s_cap + slot_i];
	}
	const int ti = unpack_cid(__float_as_uint(hi_i.w));
	const int gi = act ? S.gst[s_ocell[w]] + (t - s_own[w]) : S.gst[s_ocell[0]];
	int cnt = act ? (int) lists.count[gi] : 0;
	const bool ovf = cnt == kListOverflow;
	if (ovf && sub == 0) {
		// the list overflowed at the build: gather this molecule from global memory
		PairSums s = gather_pairs<!kFP64>(gi, rx, ry, rz, cid, cstart, bx.g, S.pd, ns, p.rc2, p.rclj2, bx.coff);
		MV += finish(kick, gi, s.F[0], s.F[1], s.F[2], rx, ry, rz, cid, lists, fx, fy, fz, status);
		U += s.U;
		W += s.W;
		NP += s.np;
		same |= s.same;
	}
	if (ovf) cnt = 0;
	const int mx = __reduce_max_sync(kFull, cnt);
	// blocks of 8 entries, one 16-byte load each, the next block loaded while this one is used;
	// this lane's blocks are sub, sub + lpm, ... (nk of them at most, the same bound in every lane)
	const uint4* my8 = reinterpret_cast<const uint4*>(lists.nbr) + gi;
	const int nb8 = (mx + 7) >> 3;
	const int nk = (nb8 + lpm - 1) / lpm;
	double Fx = 0.0, Fy = 0.0, Fz = 0.0;
	int anp = 0;
	// a prune step: kept entries go through this thread's ring and leave it in blocks of 8, the
	// lane's k-th block at inner block sub + k lpm (the blocks it would read at this split)
	int kept = 0, done = 0;
	uint4* const pdst = kPrune ? reinterpret_cast<uint4*>(po.nbr) + gi : nullptr;
	// branch-free: every entry is stored at the next free place, which only a kept entry takes
	// (at most 15 entries are unwritten, so the next free place is never one of them)
	auto keep = [&](unsigned e, bool k) {
		ring[(kept & (kPruneRing - 1)) * kThreads] = (unsigned short) e;
		kept += k ? 1 : 0;
	};
	auto flush = [&]() {
		unsigned v[4];
#pragma unroll
		for (int q = 0; q < 4; q++)
			v[q] = (unsigned) ring[((done + 2 * q) & (kPruneRing - 1)) * kThreads] |
			       ((unsigned) ring[((done + 2 * q + 1) & (kPruneRing - 1)) * kThreads] << 16);
		pdst[(int64_t) (sub + (done >> 3) * lpm) * lists.n] = make_uint4(v[0], v[1], v[2], v[3]);
		done += 8;
	};
	uint4 nxt = sub < nb8 ? my8[(int64_t) sub * lists.n] : make_uint4(0u, 0u, 0u, 0u);
	if (kFP64) {
		double ax[2] = {0, 0}, ay[2] = {0, 0}, az[2] = {0, 0}, au[2] = {0, 0}, aw[2] = {0, 0};
		for (int k = 0; k < nk; k++) {
			const int b = sub + k * lpm;
			const uint4 cur = nxt;
			if (b + lpm < nb8) nxt = my8[(int64_t) (b + lpm) * lists.n];
			const unsigned e[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
			for (int u = 0; u < 8; u++) {
				const int kk = 8 * b + u;
				const unsigned raw = (e[u >> 1] >> (16 * (u & 1))) & 0xffffu;
				const int j = min((int) raw, p.s_cap - 1);
				// (a pruned list may hold sentinel slots before its end)
				if (kk < cnt && raw < (unsigned) p.s_cap) lj64<kSingle>(p, xi, yi, zi, ti, ns, j, S, ax[u & 1], ay[u & 1], az[u & 1], au[u & 1],
				                            aw[u & 1], anp, same);
				if (kPrune) {
					// the prune test on the staged hi parts (rp2f covers the lo parts)
					const float4 hj = S.hi[j];
					const float d0 = hi_i.x - hj.x, d1 = hi_i.y - hj.y, d2 = hi_i.z - hj.z;
					keep((unsigned) j, kk < cnt && fmaf(d0, d0, fmaf(d1, d1, d2 * d2)) < po.rp2f);
				}
			}
			if (kPrune && kept - done >= 8) flush();
		}
		Fx += ax[0] + ax[1];
		Fy += ay[0] + ay[1];
		Fz += az[0] + az[1];
		U += au[0] + au[1];
		W = __dadd_rn(W, __dadd_rn(aw[0], aw[1]));
	} else {
		// FP32, branch-free. Per coordinate e = fma(m_i - m_j, step, hi_i - hi_j) with m = 2^23 +
		// the 9-bit lo field (exact integer difference, one rounding). Single-species runs sum
		// fac/eps24, s6 (s6 - 1) and s6 (2 s6 - 1) and apply eps24 and shift6 per molecule.
		const unsigned wi = __float_as_uint(hi_i.w);
		const float mix = __uint_as_float(0x4B000000u | (wi & 511u));
		const float miy = __uint_as_float(0x4B000000u | ((wi >> 9) & 511u));
		const float miz = __uint_as_float(0x4B000000u | ((wi >> 18) & 511u));
		const int nblk = (cnt + 7) >> 3;
		const unsigned sent2 = (unsigned) p.s_cap | ((unsigned) p.s_cap << 16);
		float ax[kListAcc], ay[kListAcc], az[kListAcc], au[kListAcc], aw[kListAcc];
#pragma unroll
		for (int a = 0; a < kListAcc; a++) ax[a] = ay[a] = az[a] = au[a] = aw[a] = 0.f;
		int nlj = 0;   // pairs inside the LJ cutoff (shift6 terms)
		// one pair in FP32 with the given cutoff decision; sign +1 adds it, -1 removes it
		auto pair32 = [&](int j, bool in, float sign) {
			const float4 hj = S.hi[j];
			const unsigned wj = __float_as_uint(hj.w);
			const float e0 = fmaf(mix - __uint_as_float(0x4B000000u | (wj & 511u)), bx.lo_step[0], hi_i.x - hj.x);
			const float e1 = fmaf(miy - __uint_as_float(0x4B000000u | ((wj >> 9) & 511u)), bx.lo_step[1], hi_i.y - hj.y);
			const float e2 = fmaf(miz - __uint_as_float(0x4B000000u | ((wj >> 18) & 511u)), bx.lo_step[2], hi_i.z - hj.z);
			const float d2f = fmaf(e0, e0, fmaf(e1, e1, e2 * e2));
			const bool lj_in = kLjIsRc ? in : (in && d2f < p.rclj2f);
			anp += in ? (int) sign : 0;
			if (!kLjIsRc) nlj += lj_in ? (int) sign : 0;
			const float inv = lj_in ? rcp_approx(d2f) : 0.f;
			float eps24 = 1.f, sig2 = sig2_1, shift6 = 0.f;
			if (!kSingle) {
				const int pk = ti * ns + unpack_cid(wj);
				eps24 = S.pf[pk];
				sig2 = S.pf[KK + pk];
				shift6 = S.pf[2 * KK + pk];
			}
			const float s2 = sig2 * inv;
			const float s6 = s2 * s2 * s2;
			const float r = eps24 * (s6 * fmaf(2.f, s6, -1.f));
			const float fac = sign * r * inv;
			ax[0] = fmaf(fac, e0, ax[0]);
			ay[0] = fmaf(fac, e1, ay[0]);
			az[0] = fmaf(fac, e2, az[0]);
			au[0] += sign * (fmaf(eps24 * s6, s6 - 1.f, 0.f) + (lj_in ? shift6 : 0.f));
			aw[0] += sign * r;
		};
		for (int k = 0; k < nk; k++) {
			const int b = sub + k * lpm;
			uint4 cur = nxt;
			if (b + lpm < nb8) nxt = my8[(int64_t) (b + lpm) * lists.n];
			if (b >= nblk) cur = make_uint4(sent2, sent2, sent2, sent2);
			bool amb = false;
#pragma unroll
			for (int u = 0; u < 8; u++) {
				int j = (int) ((list_word(cur, u >> 1) >> (16 * (u & 1))) & 0xffffu);
				if (kClampJ) j = min(j, p.s_cap);   // a padding entry is the caller's sentinel slot
				const float4 hj = S.hi[j];
				const unsigned wj = __float_as_uint(hj.w);
				const float h0 = hi_i.x - hj.x, h1 = hi_i.y - hj.y, h2 = hi_i.z - hj.z;  // exact
				const float g0 = mix - __uint_as_float(0x4B000000u | (wj & 511u));
				const float g1 = miy - __uint_as_float(0x4B000000u | ((wj >> 9) & 511u));
				const float g2 = miz - __uint_as_float(0x4B000000u | ((wj >> 18) & 511u));
				const float e0 = fmaf(g0, bx.lo_step[0], h0);
				const float e1 = fmaf(g1, bx.lo_step[1], h1);
				const float e2 = fmaf(g2, bx.lo_step[2], h2);
				const float d2f = fmaf(e0, e0, fmaf(e1, e1, e2 * e2));
				const bool in = d2f < p.rc2f;
				if (kPrune) keep((unsigned) j, d2f < po.rp2f);   // padding is far: never kept
				// within a few ulp of rc: decided after the block as the FP64 computation does
				amb |= fabsf(d2f - p.rc2f) <= p.band;
				anp += in ? 1 : 0;
				const bool lj_in = kLjIsRc ? in : (in && d2f < p.rclj2f);
				if (!kLjIsRc) nlj += lj_in ? 1 : 0;
				const float inv = lj_in ? rcp_approx(d2f) : 0.f;
				const int a = u % kListAcc;
				if (kSingle) {
					const float s2 = sig2_1 * inv;
					const float s6 = s2 * s2 * s2;
					const float r = s6 * fmaf(2.f, s6, -1.f);
					const float facp = r * inv;
					ax[a] = fmaf(facp, e0, ax[a]);
					ay[a] = fmaf(facp, e1, ay[a]);
					az[a] = fmaf(facp, e2, az[a]);
					au[a] = fmaf(s6, s6 - 1.f, au[a]);
					aw[a] += r;
				} else {
					const int pk = ti * ns + unpack_cid(wj);
					const float eps24 = S.pf[pk], sig2 = S.pf[KK + pk], shift6 = S.pf[2 * KK + pk];
					const float s2 = sig2 * inv;
					const float s6 = s2 * s2 * s2;
					const float r = eps24 * (s6 * fmaf(2.f, s6, -1.f));
					const float fac = r * inv;
					ax[a] = fmaf(fac, e0, ax[a]);
					ay[a] = fmaf(fac, e1, ay[a]);
					az[a] = fmaf(fac, e2, az[a]);
					au[a] = fmaf(eps24 * s6, s6 - 1.f, au[a]) + (lj_in ? shift6 : 0.f);
					aw[a] += r;
				}
			}
			if (kPrune && kept - done >= 8) flush();
			if (__any_sync(kFull, amb)) {
				// rare: pairs within a few ulp of rc whose FP64 decision differs from the FP32 one
#pragma unroll 1
				for (int u = 0; u < 8; u++) {
					int j = (int) ((list_word(cur, u >> 1) >> (16 * (u & 1))) & 0xffffu);
					if (kClampJ) j = min(j, p.s_cap);
					const float4 hj = S.hi[j];
					const unsigned wj = __float_as_uint(hj.w);
					const float e0 = fmaf(mix - __uint_as_float(0x4B000000u | (wj & 511u)), bx.lo_step[0], hi_i.x - hj.x);
					const float e1 = fmaf(miy - __uint_as_float(0x4B000000u | ((wj >> 9) & 511u)), bx.lo_step[1], hi_i.y - hj.y);
					const float e2 = fmaf(miz - __uint_as_float(0x4B000000u | ((wj >> 18) & 511u)), bx.lo_step[2], hi_i.z - hj.z);
					const float d2f = fmaf(e0, e0, fmaf(e1, e1, e2 * e2));
					if (fabsf(d2f - p.rc2f) <= p.band) {
						const bool in_f = d2f < p.rc2f;
						const bool in_d = exact_cut(S, p.rc2, j, gi, rx, ry, rz);
						if (in_f != in_d) pair32(j, true, in_d ? 1.f : -1.f);
					}
				}
			}
			if ((k & 7) == 7 || k + 1 == nk) {
				// fold the FP32 partial sums of up to 64 entries into the FP64 accumulators
				const double sc = kSingle ? (double) eps24_1 : 1.0;
				Fx += sc * acc_sum(ax);
				Fy += sc * acc_sum(ay);
				Fz += sc * acc_sum(az);
				U += sc * acc_sum(au);
				W += sc * acc_sum(aw);
#pragma unroll
				for (int a = 0; a < kListAcc; a++) ax[a] = ay[a] = az[a] = au[a] = aw[a] = 0.f;
			}
		}
		if (kSingle) U += (double) shift6_1 * (double) (kLjIsRc ? anp : nlj);
		if (!(Fx == Fx && Fy == Fy && Fz == Fz) && act && !ovf) {
			// a zero distance gives 0 * inf: report it as the reference does (same position)
			for (int k = 0; k < cnt; k++) {
				const int j = lists.nbr[(((int64_t) (k >> 3) * lists.n + gi) << 3) + (k & 7)];
				const float4 hj = S.hi[min(j, p.s_cap)];
				const unsigned pos_bits = (1u << 27) - 1u;   // the lo fields, not the component id
				if (hj.x == hi_i.x && hj.y == hi_i.y && hj.z == hi_i.z &&
				    ((__float_as_uint(hj.w) ^ wi) & pos_bits) == 0u && j != slot_i)
					same = true;
			}
		}
	}
	NP += (double) anp;
	if (kPrune) {
		// each lane's last block padded with the sentinel slot; the list ends after the molecule's
		// last written block, and a lane's blocks below that end which it did not fill hold
		// sentinels only (the evaluation reads them as far away)
		if (kept > done) {
			for (int k = kept; k < done + 8; k++) ring[(k & (kPruneRing - 1)) * kThreads] = (unsigned short) lists.sentinel;
			flush();
		}
		int end = done > 0 ? sub + ((done >> 3) - 1) * lpm + 1 : 0;
		for (int o = 1; o < lpm; o <<= 1) end = max(end, __shfl_xor_sync(kFull, end, o));
		const unsigned s2 = (unsigned) lists.sentinel | ((unsigned) lists.sentinel << 16);
		for (int b = sub + (done >> 3) * lpm; b < end; b += lpm) pdst[(int64_t) b * lists.n] = make_uint4(s2, s2, s2, s2);
		if (act && sub == 0) po.count[gi] = ovf ? kListOverflow : (unsigned short) (8 * end);
	}
	// the molecule's force: its lanes' partial sums in a fixed order
	for (int o = 1; o < lpm; o <<= 1) {
		Fx += __shfl_xor_sync(kFull, Fx, o);
		Fy += __shfl_xor_sync(kFull, Fy, o);
		Fz += __shfl_xor_sync(kFull, Fz, o);
	}
	if (act && !ovf && sub == 0) MV += finish(kick, gi, Fx, Fy, Fz, rx, ry, rz, cid, lists, fx, fy, fz, status);
}

// Forces of brick `brick` from the neighbour lists that build_lists made on the same cell
// structure, at the current positions: staging as in pairs, then the molecules of the brick's
// own cells, 32 per warp regardless of their cell, each evaluate their list with the exact cutoff.
// Chunks of 64 entries are summed in FP32 and added to FP64 accumulators.
// Shared memory: layout(s_cap, kFP64, 0, false) (no filter lists, no half-precision copy).
// kPrune: a prune step (the build lists in, the inner lists out through po).
template <bool kFP64, bool kSingle, bool kLjIsRc, bool kWide = true, bool kPrune = false>
__device__ __forceinline__ void list_pairs(const Const& p, const Box& bx, int brick, int64_t slot,
                                           unsigned char* smem, const double* rx, const double* ry, const double* rz,
                                           const int32_t* cid, const int32_t* cstart, double* fx, double* fy,
                                           double* fz, double* partials, int* status, const Lists lists,
                                           const Kick& kick, const PruneOut& po = PruneOut{}) {
	const SmemLayout L = layout(p.s_cap, kFP64, 0, false);
	const Smem S = views(smem, L);
	const int tid = threadIdx.x, warp = tid >> 5;
	const int ns = p.ns;
	const bool staged = stage<kFP64, false, kWide>(p, bx, brick, S, rx, ry, rz, cid, cstart);
	__shared__ int s_own[9], s_ocell[8];
	if (tid == 0) {
		// sentinel slot: far from every molecule (entries past a list's end point to it)
		S.hi[p.s_cap] = make_float4(1e15f, 1e15f, 1e15f, __uint_as_float((256u << 18) | (256u << 9) | 256u));
		int acc = 0;
		for (int w = 0; w < 8; w++) {
			int ic;
			const bool ok = own_cell(bx, brick, w, ic);
			s_own[w] = acc;
			s_ocell[w] = ic;
			acc += ok ? S.cnt[ic] : 0;
		}
		s_own[8] = acc;
	}
	__syncthreads();
	const int n_own = s_own[8];
	double U = 0.0, W = 0.0, NP = 0.0, MV = 0.0;
	bool same = false;
	if (!staged) {
		// over capacity: gather from global memory
		for (int t = tid; t < n_own; t += kThreads) {
			int w = 0;
			while (w < 7 && s_own[w + 1] <= t) w++;
			const int gi = S.gst[s_ocell[w]] + (t - s_own[w]);
			PairSums s = gather_pairs<!kFP64>(gi, rx, ry, rz, cid, cstart, bx.g, S.pd, ns, p.rc2, p.rclj2, bx.coff);
			MV += finish(kick, gi, s.F[0], s.F[1], s.F[2], rx, ry, rz, cid, lists, fx, fy, fz, status);
			U += s.U;
			W += s.W;
			NP += s.np;
			same |= s.same;
		}
	} else {
		// rounds of up to 256 molecules: the first as full warps of 32 (the fewest warp
		// instructions), a later one spread over every warp, g consecutive molecules with lpm lanes
		// each (lpm * g <= 32), so that no warp is left alone with a few long lists
		for (int base = 0; base < n_own; base += kThreads) {
			const int m = min(kThreads, n_own - base);
			const int g = base == 0 ? 32 : (m + kWarps - 1) / kWarps;
			const int lpm = lanes_per_molecule(g);
			const int w0 = base + warp * g, w1 = min(w0 + g, base + m);
			if (w0 < w1)
				list_chunk<kFP64, kSingle, kLjIsRc, false, kPrune>(p, bx, S, s_own, s_ocell, w0, w1, lpm, rx, ry, rz, cid,
				                                                   cstart, fx, fy, fz, status, lists, kick, U, W, NP,
				                                                   MV, same, po,
				                                                   reinterpret_cast<unsigned short*>(smem + L.total) + tid);
		}
	}
	if (same) atomicOr(status, kStatusSamePosition);
	block_sum3_at(U, W, NP, partials, slot, MV);
}

// A sparse brick (see kSparseCap) by one warp, in its own shared-memory area laid out as
// layout(kSparseCap, kFP64, 0, false) plus 17 ints (own-cell prefix and cells): staging of the 4x4x4
// region flattened over its molecules (cell found by bisection of the staged-cell starts), then
// list_chunk; U, W, pair count to partials[brick]. Warp-level synchronisation only.
__host__ __device__ inline size_t sparse_warp_bytes(bool fp64) {
	return align16(layout(kSparseCap, fp64, 0, false).total + sizeof(int) * 17);
}

template <bool kFP64, bool kSingle, bool kLjIsRc>
__device__ __forceinline__ void list_pairs_warp(const Const& p, const Box& bx, int brick, unsigned char* ws,
                                                const double* rx, const double* ry, const double* rz,
                                                const int32_t* cid, const int32_t* cstart, double* fx, double* fy,
                                                double* fz, double* partials, int* status, const Lists& lists,
                                                const Kick& kick) {
	const SmemLayout L = layout(kSparseCap, kFP64, 0, false);
	const Smem S = views(ws, L);
	int* own = reinterpret_cast<int*>(ws + L.total);
	const int lane = threadIdx.x & 31;
	const Grid& g = bx.g;
	const int bc[3] = {brick % bx.nb[0], (brick / bx.nb[0]) % bx.nb[1], brick / (bx.nb[0] * bx.nb[1])};
	for (int c = lane; c < 64; c += 32) {
		const int l[3] = {c & 3, (c >> 2) & 3, c >> 4};
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
			S.csh[3 * c + d] = sh;
			const double cbr = (2 * bc[d] + 1) * g.cell_length[d];
			S.ck[3 * c + d] = (sh - cbr) + (double) bx.frame_c[d];
		}
		const int gcell = bx.coff + (gc[2] * g.nc[1] + gc[1]) * g.nc[0] + gc[0];
		const int st = cstart[gcell];
		S.gst[c] = st;
		S.cnt[c] = max(0, cstart[gcell + 1] - st);
	}
	__syncwarp();
	{
		const int a = S.cnt[2 * lane], b = S.cnt[2 * lane + 1];
		int inc = a + b;
		for (int o = 1; o < 32; o <<= 1) {
			const int y = __shfl_up_sync(kFull, inc, o);
			if (lane >= o) inc += y;
		}
		const int excl = inc - (a + b);
		S.cs[2 * lane] = excl;
		S.cs[2 * lane + 1] = excl + a;
		if (lane == 31) S.cs[64] = inc;
	}
	__syncwarp();
	const int total = S.cs[64];
	const bool staged = total <= kSparseCap;
	if (staged) {
		for (int t = lane; t < total; t += 32) {
			int lo = 0, hi = 63;
			while (lo < hi) {
				const int mid = (lo + hi + 1) >> 1;
				if (S.cs[mid] <= t)
					lo = mid;
				else
					hi = mid - 1;
			}
			const int gi = S.gst[lo] + (t - S.cs[lo]);
			const double x = rx[gi], y = ry[gi], z = rz[gi];
			const double Xd = __dadd_rn(x, S.ck[3 * lo]), Yd = __dadd_rn(y, S.ck[3 * lo + 1]);
			const double Zd = __dadd_rn(z, S.ck[3 * lo + 2]);
			const float X = __double2float_rn(Xd), Y = __double2float_rn(Yd), Z = __double2float_rn(Zd);
			const unsigned w = pack_lo(__double2float_rn(Xd - (double) X), __double2float_rn(Yd - (double) Y),
			                           __double2float_rn(Zd - (double) Z), cid[gi], bx);
			S.hi[t] = make_float4(X, Y, Z, __uint_as_float(w));
			if (kFP64) {
				S.img[t] = __dadd_rn(x, S.csh[3 * lo]);
				S.img[kSparseCap + t] = __dadd_rn(y, S.csh[3 * lo + 1]);
				S.img[2 * kSparseCap + t] = __dadd_rn(z, S.csh[3 * lo + 2]);
			}
		}
	}
	if (lane == 0) {
		int acc = 0;
		for (int w = 0; w < 8; w++) {
			int ic;
			const bool ok = own_cell(bx, brick, w, ic);
			own[w] = acc;
			own[9 + w] = ic;
			acc += ok ? S.cnt[ic] : 0;
		}
		own[8] = acc;
	}
	__syncwarp();
	const int n_own = own[8];
	double U = 0.0, W = 0.0, NP = 0.0, MV = 0.0;
	bool same = false;
	if (staged) {
		for (int t0 = 0; t0 < n_own; t0 += 32) {
			const int g = min(32, n_own - t0);
			list_chunk<kFP64, kSingle, kLjIsRc, true>(p, bx, S, own, own + 9, t0, t0 + g, lanes_per_molecule(g), rx, ry,
			                                          rz, cid, cstart, fx, fy, fz, status, lists, kick, U, W, NP, MV,
			                                          same);
		}
	} else {
		for (int t = lane; t < n_own; t += 32) {
			int w = 0;
			while (w < 7 && own[w + 1] <= t) w++;
			const int gi = S.gst[own[9 + w]] + (t - own[w]);
			PairSums ps = gather_pairs<!kFP64>(gi, rx, ry, rz, cid, cstart, g, S.pd, p.ns, p.rc2, p.rclj2, bx.coff);
			MV += finish(kick, gi, ps.F[0], ps.F[1], ps.F[2], rx, ry, rz, cid, lists, fx, fy, fz, status);
			U += ps.U;
			W += ps.W;
			NP += ps.np;
			same |= ps.same;
		}
	}
	if (same) atomicOr(status, kStatusSamePosition);
	U = warp_sum(U);
	W = warp_sum(W);
	NP = warp_sum(NP);
	MV = warp_sum(MV);
	if (lane == 0) {
		partials[4 * (int64_t) brick + 0] = U;
		partials[4 * (int64_t) brick + 1] = W;
		partials[4 * (int64_t) brick + 2] = NP;
		partials[4 * (int64_t) brick + 3] = MV;
	}
}

}  // namespace brick
}  // namespace mdgpu
