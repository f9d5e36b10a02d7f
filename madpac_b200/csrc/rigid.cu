// Rigid multi-centre LJ molecules: the container, pair handler and Leapfrog of MarDyn for molecules
// of several LJ centres (paths relative to madpac/mardyn/).
//
// A rigid context wraps a single-box context for what does not depend on the molecules' shape: the
// particle arrays, the LinkedCells binning and cell sort of the molecule centres (launch_bin, the
// periodic wrap of DomainDecompDummy::exchangeMolecules), and the status word. What the centres add
// lives here:
//
// * orientation q (4), angular momentum D (3, space frame) and torque M (3) of every molecule, kept
//   in the caller's order (index uidx of the sorted arrays), so the cell sort never moves them;
// * k_rigid_sites: Molecule::upd_cache (molecules/Molecule.cpp:161-190): each centre's offset
//   d = q.rotateinv(site) (Quaternion.cpp:50-66) once per force evaluation, stored per sorted
//   molecule, centre-major (d[(s*3 + k)*n + i]);
// * k_rigid_pairs: the LJ block and the charge-charge block of PotForce (molecules/potforce.h:319-386;
//   PotForce2Charge, :244-253: u = q_i q_j sqrt(1/r^2), f = u/r^2 drs, UpotXpoles) for every molecule pair
//   whose centres are closer than rc (strict, particleContainer/BlockTraverse.cpp:155), every centre
//   pair evaluated when dd < rcLJ^2: drs = (drm + d_i) - d_j (SiteSiteDistance, potforce.h:26-31),
//   PotForceLJ (potforce.h:41-53), u += shift6, Upot6LJ += u, Virial += drm.f; forces summed per
//   centre, the molecule's force and torque formed from them as Molecule::calcFM does
//   (Molecule.cpp:386-411). One thread per molecule gathers over the 27 cells around it (each pair
//   seen from both sides, halved at the end: no atomics, the same sums run to run), first listing
//   the accepted partners, then evaluating them; the site-pair parameters of Comp2Param::initialize
//   (molecules/Comp2Param.cpp:28-115) in shared memory;
// * k_rigid_pre / k_rigid_post: Molecule::upd_preF and upd_postF (Molecule.cpp:128-159, 193-216)
//   with the quaternion algebra of Quaternion.cpp (rotate, differentiate, normalisation) and the
//   sums m v^2 and I w^2 of Leapfrog::transition2to3 (integrators/Leapfrog.cpp:52-99).
//
// MDGPU_FP64 evaluates everything in double with the reference's operation order and no
// contraction; MDGPU_MIXED evaluates the centre pairs of a molecule pair in float (from the double
// centre distance) and adds their sums to double accumulators once per molecule pair.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "md_internal.h"
#include "reduce.cuh"

namespace mdgpu {

constexpr int kMaxSites = MDGPU_MAX_SITES;            // LJ centres per component
constexpr int kMaxSiteTotal = MDGPU_MAX_SITE_TOTAL;   // LJ centres over all components
constexpr int kRigidThreads = kReduceBlock;

// Site tables of a rigid context (device copy read by the kernels).
struct RigidParams {
	int nc, nsite_total, ns_max;
	int nsites[kMaxSpecies];               // LJ centres + charges of component c
	int nlj[kMaxSpecies];                  // its LJ centres (sites 0..nlj-1; charges, dipoles, quadrupoles follow)
	double charge[kMaxSiteTotal];          // q of the charge sites (0 for the others)
	int type[kMaxSiteTotal];               // 0 LJ centre, 1 charge, 2 dipole, 3 quadrupole
	double strength[kMaxSiteTotal];        // q, |my| or |Q|
	double e_body[kMaxSiteTotal][3];       // orientation of a dipole or quadrupole (body frame, as given)
	double eps_rf_inv_rc3;                 // 2 (epsRF - 1) / (rc^3 (2 epsRF + 1)) (Comp2Param.cpp:178)
	int oriented;                          // any dipole or quadrupole
	int base[kMaxSpecies];                 // first centre of component c in the site tables
	double site[kMaxSiteTotal][3];         // body-frame centre positions
	double mass[kMaxSpecies];
	double I[kMaxSpecies][3], invI[kMaxSpecies][3];
	double rc2, rclj2;
	// Comp2Param stream entries per ordered pair of centres (a, b), index a * kMaxSiteTotal + b
	double eps24[kMaxSiteTotal * kMaxSiteTotal];
	double sig2[kMaxSiteTotal * kMaxSiteTotal];
	double shift6[kMaxSiteTotal * kMaxSiteTotal];
};

namespace {

inline int64_t nblocks(int64_t n) { return (n + kRigidThreads - 1) / kRigidThreads; }

// ---- quaternion algebra (Quaternion.cpp), in double without contraction -------------------------

struct Quat {
	double w, x, y, z;
};

// Quaternion::rotate: space frame -> body frame
__device__ __forceinline__ void q_rotate(const Quat& q, const double d[3], double out[3]) {
	const double ww = __dmul_rn(q.w, q.w), xx = __dmul_rn(q.x, q.x), yy = __dmul_rn(q.y, q.y),
	             zz = __dmul_rn(q.z, q.z);
	const double xy = __dmul_rn(q.x, q.y), zw = __dmul_rn(q.z, q.w), xz = __dmul_rn(q.x, q.z),
	             yw = __dmul_rn(q.y, q.w);
	out[0] = __dadd_rn(__dadd_rn(__dmul_rn(__dsub_rn(__dsub_rn(__dadd_rn(ww, xx), yy), zz), d[0]),
	                             __dmul_rn(__dmul_rn(2., __dadd_rn(xy, zw)), d[1])),
	                   __dmul_rn(__dmul_rn(2., __dsub_rn(xz, yw)), d[2]));
	const double yz = __dmul_rn(q.y, q.z), xw = __dmul_rn(q.x, q.w);
	out[1] = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(2., __dsub_rn(xy, zw)), d[0]),
	                             __dmul_rn(__dsub_rn(__dadd_rn(__dsub_rn(ww, xx), yy), zz), d[1])),
	                   __dmul_rn(__dmul_rn(2., __dadd_rn(yz, xw)), d[2]));
	out[2] = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(2., __dadd_rn(xz, yw)), d[0]),
	                             __dmul_rn(__dmul_rn(2., __dsub_rn(yz, xw)), d[1])),
	                   __dmul_rn(__dadd_rn(__dsub_rn(__dsub_rn(ww, xx), yy), zz), d[2]));
}

// Quaternion::rotateinv: body frame -> space frame
__device__ __forceinline__ void q_rotate_inv(const Quat& q, const double d[3], double out[3]) {
	const double ww = __dmul_rn(q.w, q.w), xx = __dmul_rn(q.x, q.x), yy = __dmul_rn(q.y, q.y),
	             zz = __dmul_rn(q.z, q.z);
	const double xy = __dmul_rn(q.x, q.y), zw = __dmul_rn(q.z, q.w), xz = __dmul_rn(q.x, q.z),
	             yw = __dmul_rn(q.y, q.w);
	out[0] = __dadd_rn(__dadd_rn(__dmul_rn(__dsub_rn(__dsub_rn(__dadd_rn(ww, xx), yy), zz), d[0]),
	                             __dmul_rn(__dmul_rn(2., __dsub_rn(xy, zw)), d[1])),
	                   __dmul_rn(__dmul_rn(2., __dadd_rn(xz, yw)), d[2]));
	const double yz = __dmul_rn(q.y, q.z), xw = __dmul_rn(q.x, q.w);
	out[1] = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(2., __dadd_rn(xy, zw)), d[0]),
	                             __dmul_rn(__dsub_rn(__dadd_rn(__dsub_rn(ww, xx), yy), zz), d[1])),
	                   __dmul_rn(__dmul_rn(2., __dsub_rn(yz, xw)), d[2]));
	out[2] = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(2., __dsub_rn(xz, yw)), d[0]),
	                             __dmul_rn(__dmul_rn(2., __dadd_rn(yz, xw)), d[1])),
	                   __dmul_rn(__dadd_rn(__dsub_rn(__dsub_rn(ww, xx), yy), zz), d[2]));
}

// Quaternion::differentiate: dq/dt for the body angular velocity w
__device__ __forceinline__ Quat q_differentiate(const Quat& q, const double w[3]) {
	Quat r;
	r.w = __dmul_rn(.5, __dsub_rn(__dsub_rn(__dmul_rn(-q.x, w[0]), __dmul_rn(q.y, w[1])), __dmul_rn(q.z, w[2])));
	r.x = __dmul_rn(.5, __dadd_rn(__dsub_rn(__dmul_rn(q.w, w[0]), __dmul_rn(q.z, w[1])), __dmul_rn(q.y, w[2])));
	r.y = __dmul_rn(.5, __dsub_rn(__dadd_rn(__dmul_rn(q.z, w[0]), __dmul_rn(q.w, w[1])), __dmul_rn(q.x, w[2])));
	r.z = __dmul_rn(.5, __dadd_rn(__dadd_rn(__dmul_rn(-q.y, w[0]), __dmul_rn(q.x, w[1])), __dmul_rn(q.w, w[2])));
	return r;
}

__device__ __forceinline__ double q_magnitude2(const Quat& q) {
	return __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(q.w, q.w), __dmul_rn(q.x, q.x)), __dmul_rn(q.y, q.y)),
	                 __dmul_rn(q.z, q.z));
}

__device__ __forceinline__ Quat q_scale(Quat q, double s) {
	q.w = __dmul_rn(q.w, s);
	q.x = __dmul_rn(q.x, s);
	q.y = __dmul_rn(q.y, s);
	q.z = __dmul_rn(q.z, s);
	return q;
}

__device__ __forceinline__ Quat q_add(Quat a, const Quat& b) {
	a.w = __dadd_rn(a.w, b.w);
	a.x = __dadd_rn(a.x, b.x);
	a.y = __dadd_rn(a.y, b.y);
	a.z = __dadd_rn(a.z, b.z);
	return a;
}

__device__ __forceinline__ Quat load_q(const double* q, int64_t n, int64_t u) {
	return Quat{q[u], q[n + u], q[2 * n + u], q[3 * n + u]};
}

__device__ __forceinline__ void store_q(double* q, int64_t n, int64_t u, const Quat& v) {
	q[u] = v.w;
	q[n + u] = v.x;
	q[2 * n + u] = v.y;
	q[3 * n + u] = v.z;
}

// ---- kernels ------------------------------------------------------------------------------------

// Molecule::upd_cache: the centres' space-frame offsets of every (sorted) molecule
// The mixed form of molecules with at most two LJ centres and no point polarities reads each
// partner from one 64-byte record (4 float4: x, y, z as doubles, the two centre offsets as floats,
// the component id), so a partner costs two or four 16-byte loads from one or two sectors instead
// of loads from ten separate arrays.
constexpr int kRecFloat4 = 4;
__device__ __forceinline__ float lo_f(double x) { return __int_as_float(__double2loint(x)); }
__device__ __forceinline__ float hi_f(double x) { return __int_as_float(__double2hiint(x)); }
__device__ __forceinline__ double dbl_of(float lo, float hi) {
	return __hiloint2double(__float_as_int(hi), __float_as_int(lo));
}

__global__ void __launch_bounds__(kRigidThreads) k_rigid_sites(int64_t n, const int32_t* __restrict__ uidx,
                                                               const int32_t* __restrict__ cid,
                                                               const double* __restrict__ q,
                                                               const RigidParams* __restrict__ P,
                                                               double* __restrict__ ds, float* __restrict__ dsf,
                                                               double* __restrict__ es, const double* __restrict__ rx,
                                                               const double* __restrict__ ry,
                                                               const double* __restrict__ rz,
                                                               float4* __restrict__ rec) {
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const Quat qi = load_q(q, n, uidx ? uidx[i] : i);   // caller order, or sorted with no map
	const int c = cid[i];
	const int ns = P->nsites[c], b = P->base[c];
	float df[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
	for (int s = 0; s < P->ns_max; s++) {
		double d[3] = {0.0, 0.0, 0.0}, e[3] = {0.0, 0.0, 0.0};
		if (s < ns) {
			const double body[3] = {P->site[b + s][0], P->site[b + s][1], P->site[b + s][2]};
			q_rotate_inv(qi, body, d);
			if (es && P->type[b + s] >= 2) q_rotate_inv(qi, P->e_body[b + s], e);
		}
		for (int k = 0; k < 3; k++) {
			if (!rec) {   // the records' variant reads only the records
				ds[(int64_t) (s * 3 + k) * n + i] = d[k];
				if (dsf) dsf[(int64_t) (s * 3 + k) * n + i] = (float) d[k];
			}
			if (es) es[(int64_t) (s * 3 + k) * n + i] = e[k];
			if (s < 2) df[3 * s + k] = (float) d[k];
		}
	}
	if (rec) {
		const double x = rx[i], y = ry[i], z = rz[i];
		float4* r = rec + (int64_t) kRecFloat4 * i;
		r[0] = make_float4(lo_f(x), hi_f(x), lo_f(y), hi_f(y));
		r[1] = make_float4(lo_f(z), hi_f(z), df[0], df[1]);
		r[2] = make_float4(df[2], df[3], df[4], df[5]);
		r[3] = make_float4(__int_as_float(c), 0.f, 0.f, 0.f);
	}
}

// ---- point dipoles and quadrupoles (molecules/potforce.h), double without contraction -----------

__device__ __forceinline__ double dm_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
	return da_(da_(dm_(a[0], b[0]), dm_(a[1], b[1])), dm_(a[2], b[2]));
}
__device__ __forceinline__ void cross3(const double a[3], const double b[3], double o[3]) {
	o[0] = ds_(dm_(a[1], b[2]), dm_(a[2], b[1]));
	o[1] = ds_(dm_(a[2], b[0]), dm_(a[0], b[2]));
	o[2] = ds_(dm_(a[0], b[1]), dm_(a[1], b[0]));
}

// PotForceChargeQuadrupole (potforce.h:256-281) / PotForceChargeDipole (:284-311): f, and m2 the
// torque on the oriented site ejj.
__device__ void charge_oriented(bool quad, const double dr[3], double dr2, const double ejj[3], double par,
                                double f[3], double m2[3], double& u) {
	const double invdr2 = __ddiv_rn(1.0, dr2);
	const double invdr = __dsqrt_rn(invdr2);
	const double costj = dm_(dot3(ejj, dr), invdr);
	double pT, fac;
	if (quad) {
		const double qQinv4dr3 = dm_(dm_(par, invdr), invdr2);
		u = dm_(qQinv4dr3, ds_(dm_(dm_(3.0, costj), costj), 1.0));
		const double pR = dm_(dm_(-3.0, u), invdr2);
		pT = dm_(dm_(dm_(6.0, costj), qQinv4dr3), invdr);
		fac = ds_(dm_(dm_(costj, pT), invdr), pR);
	} else {
		const double uInvcostj = dm_(par, invdr2);
		u = dm_(uInvcostj, costj);
		pT = dm_(uInvcostj, invdr);
		fac = dm_(dm_(dm_(3.0, u), invdr), invdr2);
	}
	for (int d = 0; d < 3; d++) f[d] = ds_(dm_(fac, dr[d]), dm_(pT, ejj[d]));
	const double mx[3] = {ds_(dm_(ejj[2], dr[1]), dm_(ejj[1], dr[2])), ds_(dm_(ejj[0], dr[2]), dm_(ejj[2], dr[0])),
	                      ds_(dm_(ejj[1], dr[0]), dm_(ejj[0], dr[1]))};
	for (int d = 0; d < 3; d++) m2[d] = dm_(pT, mx[d]);
}

// PotForce2Dipole (kind 0, :66-113), PotForce2Quadrupole (1, :127-172), PotForceDiQuadrupole
// (2, :186-229, dipole eii, quadrupole ejj): f, m1 (torque on eii), m2 (on ejj), u, MyRF increment.
__device__ void two_oriented(int kind, const double dr[3], double dr2, const double eii[3], const double ejj[3],
                             double par, double rffac, double f[3], double m1[3], double m2[3], double& u,
                             double& rf) {
	const double invdr2 = __ddiv_rn(1., dr2);
	const double invdr1 = __dsqrt_rn(invdr2);
	const double costi = dm_(dot3(eii, dr), invdr1);
	const double costj = dm_(dot3(ejj, dr), invdr1);
	const double cosgij = dot3(eii, ejj);
	double pR, pTi, pTj, pG;
	rf = 0.0;
	if (kind == 0) {
		const double myfac = dm_(dm_(par, invdr2), invdr1);
		u = dm_(myfac, ds_(cosgij, dm_(dm_(3., costi), costj)));
		rf = -dm_(rffac, cosgij);
		pR = dm_(dm_(-3., u), invdr2);
		pTi = dm_(dm_(dm_(-myfac, 3.), costj), invdr1);
		pTj = dm_(dm_(dm_(-myfac, 3.), costi), invdr1);
		pG = myfac;
	} else if (kind == 1) {
		const double qfac = dm_(dm_(dm_(par, invdr2), invdr2), invdr1);
		const double c2i = dm_(costi, costi), c2j = dm_(costj, costj);
		const double term = ds_(cosgij, dm_(dm_(5., costi), costj));
		u = dm_(qfac, da_(ds_(ds_(1., dm_(5., da_(c2i, c2j))), dm_(dm_(15., c2i), c2j)), dm_(dm_(2., term), term)));
		pR = dm_(dm_(-5., u), invdr2);
		pTi = dm_(dm_(dm_(-qfac, 10.), da_(da_(costi, dm_(dm_(3., costi), c2j)), dm_(dm_(2., costj), term))), invdr1);
		pTj = dm_(dm_(dm_(-qfac, 10.), da_(da_(costj, dm_(dm_(3., c2i), costj)), dm_(dm_(2., costi), term))), invdr1);
		pG = dm_(dm_(qfac, 4.), term);
	} else {
		const double myqfac = dm_(dm_(par, invdr2), invdr2);
		const double c2j = dm_(costj, costj);
		u = dm_(myqfac, da_(dm_(-costi, ds_(dm_(5., c2j), 1.)), dm_(dm_(2., cosgij), costj)));
		pR = dm_(dm_(-4., u), invdr2);
		pTi = dm_(dm_(myqfac, da_(dm_(-5., c2j), 1.)), invdr1);
		pTj = dm_(dm_(dm_(myqfac, 2.), da_(dm_(dm_(-5., costi), costj), cosgij)), invdr1);
		pG = dm_(dm_(myqfac, 2.), costj);
	}
	const double fac = da_(-pR, dm_(da_(dm_(costi, pTi), dm_(costj, pTj)), invdr1));
	for (int d = 0; d < 3; d++) f[d] = ds_(ds_(dm_(fac, dr[d]), dm_(pTi, eii[d])), dm_(pTj, ejj[d]));
	double eiXej[3], eXr[3];
	cross3(eii, ejj, eiXej);
	cross3(eii, dr, eXr);
	const double g1 = kind == 0 ? da_(-pG, rffac) : -pG;
	for (int d = 0; d < 3; d++) m1[d] = da_(dm_(-pTi, eXr[d]), dm_(g1, eiXej[d]));
	cross3(ejj, dr, eXr);
	const double g2 = kind == 0 ? ds_(pG, rffac) : pG;
	for (int d = 0; d < 3; d++) m2[d] = da_(dm_(-pTj, eXr[d]), dm_(g2, eiXej[d]));
}

// One point-polarity site pair of PotForce(mi = i, mj = j) (potforce.h:372-542; charge-charge is
// evaluated by the caller): the force on i's site (fi), the direct torque on i (mi), u, the
// molecule pair's virial term (w, with the block's sign) and the MyRF increment. drm from j to i.
__device__ void polar_pair(int ti, int tj, const double drm[3], const double di[3], const double dj[3],
                           const double ei[3], const double ej[3], double si, double sj, double rfc, double fi[3],
                           double mi[3], double& u, double& w, double& rf) {
	double dr[3], f[3], mo[3];
	const bool minus = (ti == 3 && tj != 3) || (ti == 2 && tj == 1);   // minusSiteSiteDistance blocks
	for (int d = 0; d < 3; d++)
		dr[d] = minus ? ds_(ds_(dj[d], drm[d]), di[d]) : ds_(da_(drm[d], di[d]), dj[d]);
	const double dr2 = dot3(dr, dr);
	mi[0] = mi[1] = mi[2] = 0.0;
	rf = 0.0;
	if (ti == 1) {                                   // Charge-Quadrupole, Charge-Dipole
		charge_oriented(tj == 3, dr, dr2, ej, tj == 3 ? dm_(dm_(0.25, si), sj) : dm_(-si, sj), f, mo, u);
	} else if (tj == 1) {                            // Quadrupole-Charge, Dipole-Charge
		charge_oriented(ti == 3, dr, dr2, ei, ti == 3 ? dm_(dm_(0.25, sj), si) : dm_(-sj, si), f, mi, u);
	} else if (ti == 3 && tj == 2) {                 // Quadrupole-Dipole: the dipole is the first argument
		two_oriented(2, dr, dr2, ej, ei, dm_(dm_(1.5, si), sj), 0.0, f, mo, mi, u, rf);
	} else {                                         // Quadrupole-Quadrupole, Dipole-Quadrupole, Dipole-Dipole
		const int kind = ti == 3 ? 1 : (tj == 3 ? 2 : 0);
		const double par = kind == 1 ? dm_(dm_(.75, si), sj) : (kind == 2 ? dm_(dm_(1.5, si), sj) : dm_(si, sj));
		two_oriented(kind, dr, dr2, ei, ej, par, kind == 0 ? dm_(par, rfc) : 0.0, f, mi, mo, u, rf);
	}
	const double sgn = minus ? -1.0 : 1.0;
	for (int d = 0; d < 3; d++) fi[d] = sgn * f[d];
	w = sgn * dot3(drm, f);
}

struct RigidOut {
	double* fx;
	double* fy;
	double* fz;
	double* M;          // caller order, M[k*n + u]
	double* partials;
	unsigned* ticket;
	double* scalars;    // [0..3] = sum LJ u, sum drm.f, pairs, sum charge u (each pair from both sides)
	int* status;
};

// Lanes per molecule of the pair kernel (consecutive lanes; a warp holds 16 consecutive molecules of
// the cell order, about two cells, so its lanes walk mostly the same candidate cells), and the
// accepted partners each lane lists per pass, in shared memory (one column per thread; the static
// 48 KB bounds the depth). Measured on the 1M-molecule 2CLJ fluid: 2 lanes 2.21 ms per step, 4 lanes
// 2.69, 8 lanes 3.46, 1 lane (40 entries, which the FCC start's 42 partners overflow) 11.9.
#ifndef MDGPU_RIGID_LANES
#define MDGPU_RIGID_LANES 2
#endif
#ifndef MDGPU_RIGID_LIST
#define MDGPU_RIGID_LIST 32
#endif
#ifndef MDGPU_RIGID_DIRECT
#define MDGPU_RIGID_DIRECT 0
#endif
// list entries evaluated as they are accepted instead of through the lane's shared-memory list
constexpr bool kDirect = MDGPU_RIGID_DIRECT != 0;
constexpr int kRigidLanes = MDGPU_RIGID_LANES;
constexpr int kRigidList = MDGPU_RIGID_LIST;
static_assert(kRigidLanes == 1 || kRigidLanes == 2 || kRigidLanes == 4 || kRigidLanes == 8, "lanes per molecule");

// kRigidLanes lanes per sorted molecule i: force and torque from every molecule of the 27 cells
// around it (lane k of the molecule takes every kRigidLanes-th candidate of each cell), in two
// phases so that the centre-pair arithmetic runs with the warp's lanes busy:
//   scan:     every candidate j is tested against rc (the exact double test of the reference); the
//             accepted ones within rcLJ go to the lane's list as j << 5 | image (the periodic image
//             of j's cell, 27 codes);
//   evaluate: the list's molecule pairs, every centre pair of each (a pass is evaluated early when
//             the list fills).
// Forces are summed per centre of i, the lanes' sums combined in a fixed order (butterfly), and the
// torque formed at the end as calcFM does (M = sum_s d_s x F_s); the virial term of a molecule pair
// is drm . (sum of its centre forces).
// kQ: 0 LJ centres only, 1 with charges, 2 with dipoles or quadrupoles as well
//
// Verlet-skin mode (vl.list non-null): the candidates are molecule i's entries of the list that
// k_rigid_build made (codes j << 5 | image, within rc + skin at the build), tested with the same
// exact double cutoff; a molecule whose list overflowed at the build (count -1) scans its 27 cells
// of the skin grid instead, which finds the same partners: since the build no molecule has moved
// more than skin/2, and the cells are at least rc + skin wide.
struct RigidLists {
	const uint32_t* list;    // cap x n, entry k of molecule i at k * n + i
	const int32_t* count;    // per molecule; -1: overflowed at the build
};

// CTAs per SM: the mixed two-centre LJ variant (the records') three (85 registers, a few spilled:
// 1.19 against 1.45 ms per step at two CTAs on the 1 M two-centre fluid), the others with up to four
// sites and no dipoles or quadrupoles two (128 registers), the rest one.
template <bool kMixed, int NS, int kQ>
__global__ void __launch_bounds__(kRigidThreads,
                                  (kMixed && NS <= 2 && kQ == 0) ? 3 : ((kQ == 2 || NS > 4) ? 1 : 2))
    k_rigid_pairs(int64_t n, const double* __restrict__ rx,
                                                               const double* __restrict__ ry,
                                                               const double* __restrict__ rz,
                                                               const int32_t* __restrict__ cid,
                                                               const int32_t* __restrict__ uidx,
                                                               const int32_t* __restrict__ start, Grid g,
                                                               const RigidParams* __restrict__ P,
                                                               const double* __restrict__ ds,
                                                               const float* __restrict__ dsf,
                                                               const double* __restrict__ es, RigidOut o,
                                                               RigidLists vl, const float4* __restrict__ rec) {
	// partners from the 64-byte records (filled by k_rigid_sites for these variants)
	constexpr bool kRec = kMixed && NS <= 2 && kQ == 0;
	constexpr int TT = kMaxSiteTotal * kMaxSiteTotal;
	__shared__ double s_e24[TT], s_sig2[TT], s_sh6[TT];
	__shared__ int s_ns[kMaxSpecies], s_nlj[kMaxSpecies], s_base[kMaxSpecies];
	__shared__ double s_q[kMaxSiteTotal], s_str[kMaxSiteTotal];
	__shared__ int s_type[kMaxSiteTotal];
	__shared__ float s_e24f[kMixed ? TT : 1], s_sig2f[kMixed ? TT : 1], s_qf[kMixed ? kMaxSiteTotal : 1];
	__shared__ uint32_t s_list[kRigidList * kRigidThreads];
	for (int k = threadIdx.x; k < TT; k += blockDim.x) {
		s_e24[k] = P->eps24[k];
		s_sig2[k] = P->sig2[k];
		s_sh6[k] = P->shift6[k];
		if constexpr (kMixed) {
			s_e24f[k] = (float) P->eps24[k];
			s_sig2f[k] = (float) P->sig2[k];
		}
	}
	if constexpr (kMixed)
		if (threadIdx.x < kMaxSiteTotal) s_qf[threadIdx.x] = (float) P->charge[threadIdx.x];
	// the records' variant: the shift6 terms of all centre pairs of a component pair, summed once
	// (every centre pair of a listed molecule pair is evaluated there: no charges, all within rcLJ)
	__shared__ double s_shpair[kRec ? kMaxSpecies * kMaxSpecies : 1];
	if constexpr (kRec)
		if (threadIdx.x < kMaxSpecies * kMaxSpecies) {
			const int ca = threadIdx.x / kMaxSpecies, cb = threadIdx.x % kMaxSpecies;
			double t = 0.0;
			if (ca < P->nc && cb < P->nc)
				for (int sa = 0; sa < P->nsites[ca]; sa++)
					for (int sb = 0; sb < P->nsites[cb]; sb++)
						t += P->shift6[(P->base[ca] + sa) * kMaxSiteTotal + P->base[cb] + sb];
			s_shpair[threadIdx.x] = t;
		}
	if (threadIdx.x < kMaxSpecies) {
		s_ns[threadIdx.x] = P->nsites[threadIdx.x];
		s_nlj[threadIdx.x] = P->nlj[threadIdx.x];
		s_base[threadIdx.x] = P->base[threadIdx.x];
	}
	if (threadIdx.x < kMaxSiteTotal) {
		s_q[threadIdx.x] = P->charge[threadIdx.x];
		s_str[threadIdx.x] = P->strength[threadIdx.x];
		s_type[threadIdx.x] = P->type[threadIdx.x];
	}
	constexpr bool oriented = kQ == 2;
	const double rfc = P->eps_rf_inv_rc3;
	__syncthreads();
	const double rc2 = P->rc2, rclj2 = P->rclj2;
	const int64_t i = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) / kRigidLanes;
	const int sub = (int) (threadIdx.x % kRigidLanes);
	double Fs[NS][3];
#pragma unroll
	for (int s = 0; s < NS; s++) Fs[s][0] = Fs[s][1] = Fs[s][2] = 0.0;
	double U = 0.0, UX = 0.0, W = 0.0, np = 0.0;
	double Md[3] = {0.0, 0.0, 0.0};   // direct torques of the dipole and quadrupole pairs (Madd)
	bool same = false;
	// centre offsets of i: double for the FP64 form, float for the mixed one (the double values are
	// read again for the torque at the end)
	double di[kMixed ? 1 : NS][3];
	float dif[kMixed ? NS : 1][3];
	int nsi = 0;
	if (i < n) {
		const double xi = rx[i], yi = ry[i], zi = rz[i];
		const int ci = cid[i];
		nsi = s_ns[ci];
		const int nlji = s_nlj[ci];
		const int bi = s_base[ci];
		if constexpr (kRec) {
			// the molecule's own centre offsets from its record (the variant writes no ds)
			const float4* r4 = rec + (int64_t) kRecFloat4 * i;
			const float4 B = r4[1], C = r4[2];
			const float o[6] = {B.z, B.w, C.x, C.y, C.z, C.w};
#pragma unroll
			for (int s = 0; s < NS; s++)
#pragma unroll
				for (int k = 0; k < 3; k++) dif[s][k] = s < nsi ? o[3 * s + k] : 0.f;
		} else {
#pragma unroll
			for (int s = 0; s < NS; s++)
#pragma unroll
				for (int k = 0; k < 3; k++) {
					const double v = s < nsi ? ds[(int64_t) (s * 3 + k) * n + i] : 0.0;
					if constexpr (kMixed)
						dif[s][k] = (float) v;
					else
						di[s][k] = v;
				}
		}
		uint32_t* list = s_list + threadIdx.x;
		int cnt = 0;

		// the molecule pairs of the list: every LJ centre pair of each (within rcLJ) and every charge
		// pair (PotForce2Charge, potforce.h:244-253)
		// one accepted molecule pair (code j << 5 | image)
		auto eval_pair = [&](uint32_t code) {
			{
				const int j = (int) (code >> 5);
				const int img = (int) (code & 31u);
				const double sx = (double) (img % 3 - 1) * g.L[0];
				const double sy = (double) ((img / 3) % 3 - 1) * g.L[1];
				const double sz = (double) (img / 9 - 1) * g.L[2];
				double xj, yj, zj;
				int cj;
				float djr[2][3];
				if constexpr (kRec) {
					const float4* r4 = rec + (int64_t) kRecFloat4 * j;
					const float4 A = r4[0], B = r4[1], C = r4[2], D = r4[3];
					xj = dbl_of(A.x, A.y);
					yj = dbl_of(A.z, A.w);
					zj = dbl_of(B.x, B.y);
					djr[0][0] = B.z;
					djr[0][1] = B.w;
					djr[0][2] = C.x;
					djr[1][0] = C.y;
					djr[1][1] = C.z;
					djr[1][2] = C.w;
					cj = __float_as_int(D.x);
				} else {
					xj = rx[j];
					yj = ry[j];
					zj = rz[j];
					cj = cid[j];
				}
				const double m0 = __dsub_rn(xi, __dadd_rn(xj, sx));
				const double m1 = __dsub_rn(yi, __dadd_rn(yj, sy));
				const double m2 = __dsub_rn(zi, __dadd_rn(zj, sz));
				// without charges the list holds only partners within rcLJ
				const bool lj =
				    !kQ || __dadd_rn(__dadd_rn(__dmul_rn(m0, m0), __dmul_rn(m1, m1)), __dmul_rn(m2, m2)) < rclj2;
				const int nsj = s_ns[cj], nljj = s_nlj[cj], bj = s_base[cj];
				double fp0 = 0.0, fp1 = 0.0, fp2 = 0.0;   // force of this molecule pair
				if constexpr (!kMixed) {
#pragma unroll
					for (int sj = 0; sj < NS; sj++) {
						if (sj >= nsj) break;
						const bool lj_j = !kQ || sj < nljj;
						if (lj_j && !lj) continue;
						const double dj0 = ds[(int64_t) (sj * 3 + 0) * n + j];
						const double dj1 = ds[(int64_t) (sj * 3 + 1) * n + j];
						const double dj2 = ds[(int64_t) (sj * 3 + 2) * n + j];
#pragma unroll
						for (int si = 0; si < NS; si++) {
							if (si >= nsi) break;
							// LJ with LJ, charge with charge (the other point-polarity pairs below)
							if (kQ && (lj_j ? si >= nlji : (s_type[bi + si] != 1 || s_type[bj + sj] != 1))) continue;
							// SiteSiteDistance: drs = drm + d_i - d_j
							const double s0 = __dsub_rn(__dadd_rn(m0, di[si][0]), dj0);
							const double s1 = __dsub_rn(__dadd_rn(m1, di[si][1]), dj1);
							const double s2 = __dsub_rn(__dadd_rn(m2, di[si][2]), dj2);
							const double dr2 =
							    __dadd_rn(__dadd_rn(__dmul_rn(s0, s0), __dmul_rn(s1, s1)), __dmul_rn(s2, s2));
							const double invdr2 = __ddiv_rn(1.0, dr2);
							double fac;
							if (lj_j) {
								const int pk = (bi + si) * kMaxSiteTotal + bj + sj;
								const double eps24 = s_e24[pk];
								double lj6 = __dmul_rn(s_sig2[pk], invdr2);
								lj6 = __dmul_rn(__dmul_rn(lj6, lj6), lj6);
								const double lj12 = __dmul_rn(lj6, lj6);
								const double lj12m6 = __dsub_rn(lj12, lj6);
								U = __dadd_rn(U, __dadd_rn(__dmul_rn(eps24, lj12m6), s_sh6[pk]));
								fac = __dmul_rn(__dmul_rn(eps24, __dadd_rn(lj12, lj12m6)), invdr2);
							} else {
								const double u = __dmul_rn(__dmul_rn(s_q[bi + si], s_q[bj + sj]), __dsqrt_rn(invdr2));
								UX = __dadd_rn(UX, u);
								fac = __dmul_rn(u, invdr2);
							}
							const double f0 = __dmul_rn(fac, s0), f1 = __dmul_rn(fac, s1), f2 = __dmul_rn(fac, s2);
							Fs[si][0] = __dadd_rn(Fs[si][0], f0);
							Fs[si][1] = __dadd_rn(Fs[si][1], f1);
							Fs[si][2] = __dadd_rn(Fs[si][2], f2);
							fp0 = __dadd_rn(fp0, f0);
							fp1 = __dadd_rn(fp1, f1);
							fp2 = __dadd_rn(fp2, f2);
						}
					}
				} else {
					const float e0 = (float) m0, e1 = (float) m1, e2 = (float) m2;
					float fs[NS][3];
#pragma unroll
					for (int si = 0; si < NS; si++) fs[si][0] = fs[si][1] = fs[si][2] = 0.0f;
					float uf = 0.0f, uq = 0.0f;
					double sh = 0.0;
#pragma unroll
					for (int sj = 0; sj < NS; sj++) {
						if (sj >= nsj) break;
						const bool lj_j = !kQ || sj < nljj;
						if (lj_j && !lj) continue;
						float dj0, dj1, dj2;
						if constexpr (kRec) {
							dj0 = djr[sj][0];
							dj1 = djr[sj][1];
							dj2 = djr[sj][2];
						} else {
							dj0 = dsf[(int64_t) (sj * 3 + 0) * n + j];
							dj1 = dsf[(int64_t) (sj * 3 + 1) * n + j];
							dj2 = dsf[(int64_t) (sj * 3 + 2) * n + j];
						}
#pragma unroll
						for (int si = 0; si < NS; si++) {
							if (si >= nsi) break;
							if (kQ && (lj_j ? si >= nlji : (s_type[bi + si] != 1 || s_type[bj + sj] != 1))) continue;
							const float s0 = e0 + dif[si][0] - dj0;
							const float s1 = e1 + dif[si][1] - dj1;
							const float s2 = e2 + dif[si][2] - dj2;
							const float dr2 = s0 * s0 + s1 * s1 + s2 * s2;
							const float inv = __fdividef(1.0f, dr2);
							float fac;
							if (lj_j) {
								const int pk = (bi + si) * kMaxSiteTotal + bj + sj;
								const float eps24 = s_e24f[pk];
								const float q2 = s_sig2f[pk] * inv;
								const float q6 = q2 * q2 * q2;
								const float q12 = q6 * q6;
								const float qm = q12 - q6;
								fac = eps24 * (q12 + qm) * inv;
								uf += eps24 * qm;
								if constexpr (!kRec) sh += s_sh6[pk];
							} else {
								const float u = s_qf[bi + si] * s_qf[bj + sj] * rsqrtf(dr2);
								uq += u;
								fac = u * inv;
							}
							fs[si][0] += fac * s0;
							fs[si][1] += fac * s1;
							fs[si][2] += fac * s2;
						}
					}
					if constexpr (kRec) {
						// the molecule pair's force and its virial term drm . f in float
						float q0 = 0.f, q1 = 0.f, q2 = 0.f;
#pragma unroll
						for (int si = 0; si < NS; si++) {
							if (si >= nsi) break;
							Fs[si][0] += (double) fs[si][0];
							Fs[si][1] += (double) fs[si][1];
							Fs[si][2] += (double) fs[si][2];
							q0 += fs[si][0];
							q1 += fs[si][1];
							q2 += fs[si][2];
						}
						U += (double) uf + s_shpair[ci * kMaxSpecies + cj];
						W += (double) (e0 * q0 + e1 * q1 + e2 * q2);
					} else {
						U += (double) uf + sh;
						UX += (double) uq;
#pragma unroll
						for (int si = 0; si < NS; si++) {
							if (si >= nsi) break;
							Fs[si][0] += (double) fs[si][0];
							Fs[si][1] += (double) fs[si][1];
							Fs[si][2] += (double) fs[si][2];
							fp0 += (double) fs[si][0];
							fp1 += (double) fs[si][1];
							fp2 += (double) fs[si][2];
						}
					}
				}
				if constexpr (oriented) {
					// pairs with a dipole or quadrupole, in double in both forms (polar_pair)
					const double drm[3] = {m0, m1, m2};
					for (int sj = nljj; sj < nsj; sj++) {
						const int tj = s_type[bj + sj];
						double dj[3], ej[3];
						for (int k = 0; k < 3; k++) {
							dj[k] = ds[(int64_t) (sj * 3 + k) * n + j];
							ej[k] = es[(int64_t) (sj * 3 + k) * n + j];
						}
#pragma unroll
						for (int si = 0; si < NS; si++) {
							if (si >= nsi) break;
							const int ti = s_type[bi + si];
							if (ti == 0 || (ti == 1 && tj == 1)) continue;
							if (ti == 1 && tj == 0) continue;
							double dii[3], eii[3], fi[3], mi[3], u, w, rf;
							for (int k = 0; k < 3; k++) {
								dii[k] = ds[(int64_t) (si * 3 + k) * n + i];
								eii[k] = es[(int64_t) (si * 3 + k) * n + i];
							}
							polar_pair(ti, tj, drm, dii, dj, eii, ej, s_str[bi + si], s_str[bj + sj], rfc, fi, mi, u, w, rf);
							Fs[si][0] = __dadd_rn(Fs[si][0], fi[0]);
							Fs[si][1] = __dadd_rn(Fs[si][1], fi[1]);
							Fs[si][2] = __dadd_rn(Fs[si][2], fi[2]);
							fp0 = __dadd_rn(fp0, fi[0]);
							fp1 = __dadd_rn(fp1, fi[1]);
							fp2 = __dadd_rn(fp2, fi[2]);
							Md[0] = __dadd_rn(Md[0], mi[0]);
							Md[1] = __dadd_rn(Md[1], mi[1]);
							Md[2] = __dadd_rn(Md[2], mi[2]);
							// ParticlePairs2PotForceAdapter::finish adds MyRF to Upot and 3 MyRF to the virial
							UX = __dadd_rn(UX, __dadd_rn(u, rf));
							W = __dadd_rn(W, __dmul_rn(3.0, rf));
						}
					}
				}
				// Virial += drm . f over the molecule pair's site pairs
				if constexpr (!kRec)
					W = __dadd_rn(W, __dadd_rn(__dadd_rn(__dmul_rn(m0, fp0), __dmul_rn(m1, fp1)), __dmul_rn(m2, fp2)));
			}
		};
		auto evaluate = [&]() {
			for (int e = 0; e < cnt; e++) eval_pair(list[e * kRigidThreads]);
			cnt = 0;
		};

		// candidate j in image img (shift sx, sy, sz): the exact cutoff test of the reference; the
		// accepted ones go to the lane's list
		auto consider = [&](int j, uint32_t img, double sx, double sy, double sz) {
			double xj, yj, zj;
			if constexpr (kRec) {
				const float4* r4 = rec + (int64_t) kRecFloat4 * j;
				const float4 A = r4[0], B = r4[1];
				xj = dbl_of(A.x, A.y);
				yj = dbl_of(A.z, A.w);
				zj = dbl_of(B.x, B.y);
			} else {
				xj = rx[j];
				yj = ry[j];
				zj = rz[j];
			}
			// the halo image of j (DomainDecompDummy.cpp:64-70, 93-99); adding 0 is exact
			const double m0 = __dsub_rn(xi, __dadd_rn(xj, sx));
			const double m1 = __dsub_rn(yi, __dadd_rn(yj, sy));
			const double m2 = __dsub_rn(zi, __dadd_rn(zj, sz));
			const double dd = __dadd_rn(__dadd_rn(__dmul_rn(m0, m0), __dmul_rn(m1, m1)), __dmul_rn(m2, m2));
			if (!(dd < rc2)) return;
			np += 1.0;
			if (dd == 0.0) same = true;
			if (!kQ && !(dd < rclj2)) return;
			const uint32_t code = ((uint32_t) j << 5) | img;
			if (kDirect && vl.list) {
				eval_pair(code);   // from a list: evaluated at once
				return;
			}
			list[cnt * kRigidThreads] = code;
			if (++cnt == kRigidList) evaluate();
		};
		const int32_t nlist = vl.list ? vl.count[i] : -1;
		if (nlist >= 0) {
			for (int e = sub; e < nlist; e += kRigidLanes) {
				const uint32_t code = vl.list[(int64_t) e * n + i];
				const uint32_t img = code & 31u;
				consider((int) (code >> 5), img, (double) ((int) (img % 3u) - 1) * g.L[0],
				         (double) ((int) ((img / 3u) % 3u) - 1) * g.L[1], (double) ((int) (img / 9u) - 1) * g.L[2]);
			}
		} else {
			int cc[3];
			const double r[3] = {xi, yi, zi};
			for (int d = 0; d < 3; d++) {
				int c = (int) floor(__ddiv_rn(__dsub_rn(r[d], g.halo_min[d]), g.cell_length[d])) - 1;
				cc[d] = c < 0 ? 0 : (c >= g.nc[d] ? g.nc[d] - 1 : c);
			}
			for (int dz = -1; dz <= 1; dz++) {
				int z = cc[2] + dz, iz = 1;
				if (z < 0) {
					z += g.nc[2];
					iz = 0;
				} else if (z >= g.nc[2]) {
					z -= g.nc[2];
					iz = 2;
				}
				const double sz = (double) (iz - 1) * g.L[2];
				for (int dy = -1; dy <= 1; dy++) {
					int y = cc[1] + dy, iy = 1;
					if (y < 0) {
						y += g.nc[1];
						iy = 0;
					} else if (y >= g.nc[1]) {
						y -= g.nc[1];
						iy = 2;
					}
					const double sy = (double) (iy - 1) * g.L[1];
					for (int dx = -1; dx <= 1; dx++) {
						int x = cc[0] + dx, ix = 1;
						if (x < 0) {
							x += g.nc[0];
							ix = 0;
						} else if (x >= g.nc[0]) {
							x -= g.nc[0];
							ix = 2;
						}
						const double sx = (double) (ix - 1) * g.L[0];
						const uint32_t img = (uint32_t) (ix + 3 * iy + 9 * iz);
						const bool shifted = img != 13u;
						const int nb = (z * g.nc[1] + y) * g.nc[0] + x;
						const int j0 = start[nb], j1 = start[nb + 1];
						for (int j = j0 + sub; j < j1; j += kRigidLanes) {
							if (j == i && !shifted) continue;
							consider(j, img, sx, sy, sz);
						}
					}
				}
			}
		}
		evaluate();
	} else {
#pragma unroll
		for (int s = 0; s < (kMixed ? 1 : NS); s++) di[s][0] = di[s][1] = di[s][2] = 0.0;
	}
	// the molecule's lanes combine their sums (the same order in every lane)
	__syncwarp();
#pragma unroll
	for (int o2 = 1; o2 < kRigidLanes; o2 <<= 1) {
#pragma unroll
		for (int s = 0; s < NS; s++)
#pragma unroll
			for (int k = 0; k < 3; k++) Fs[s][k] = __dadd_rn(Fs[s][k], __shfl_xor_sync(0xffffffffu, Fs[s][k], o2));
		U = __dadd_rn(U, __shfl_xor_sync(0xffffffffu, U, o2));
		UX = __dadd_rn(UX, __shfl_xor_sync(0xffffffffu, UX, o2));
		if constexpr (kQ == 2)
			for (int k = 0; k < 3; k++) Md[k] = __dadd_rn(Md[k], __shfl_xor_sync(0xffffffffu, Md[k], o2));
		W = __dadd_rn(W, __shfl_xor_sync(0xffffffffu, W, o2));
		np += __shfl_xor_sync(0xffffffffu, np, o2);
	}
	if (sub != 0) U = UX = W = np = 0.0;
	if (i < n && sub == 0) {
		double F[3] = {0.0, 0.0, 0.0}, Mt[3] = {0.0, 0.0, 0.0};
		// Molecule::calcFM: F = sum F_s, M = sum d_s x F_s
#pragma unroll
		for (int s = 0; s < NS; s++) {
			if (s >= nsi) break;
			F[0] = __dadd_rn(F[0], Fs[s][0]);
			F[1] = __dadd_rn(F[1], Fs[s][1]);
			F[2] = __dadd_rn(F[2], Fs[s][2]);
			double d[3];
			if constexpr (kRec) {
				for (int k = 0; k < 3; k++) d[k] = (double) dif[s][k];   // the float offsets of the record
			} else if constexpr (kMixed) {
				for (int k = 0; k < 3; k++) d[k] = ds[(int64_t) (s * 3 + k) * n + i];
			} else {
				d[0] = di[s][0];
				d[1] = di[s][1];
				d[2] = di[s][2];
			}
			Mt[0] = __dadd_rn(Mt[0], __dsub_rn(__dmul_rn(d[1], Fs[s][2]), __dmul_rn(d[2], Fs[s][1])));
			Mt[1] = __dadd_rn(Mt[1], __dsub_rn(__dmul_rn(d[2], Fs[s][0]), __dmul_rn(d[0], Fs[s][2])));
			Mt[2] = __dadd_rn(Mt[2], __dsub_rn(__dmul_rn(d[0], Fs[s][1]), __dmul_rn(d[1], Fs[s][0])));
		}
		for (int k = 0; k < 3; k++) Mt[k] = __dadd_rn(Mt[k], Md[k]);
		o.fx[i] = F[0];
		o.fy[i] = F[1];
		o.fz[i] = F[2];
		const int64_t u = uidx ? uidx[i] : i;
		o.M[u] = Mt[0];
		o.M[n + u] = Mt[1];
		o.M[2 * n + u] = Mt[2];
		const bool bad = !(isfinite(F[0]) && isfinite(F[1]) && isfinite(F[2]) && isfinite(Mt[0]) &&
		                   isfinite(Mt[1]) && isfinite(Mt[2]));
		if (bad) atomicOr(o.status, kStatusNonFinite);
	}
	if (same) atomicOr(o.status, kStatusSamePosition);
	block_sum3_at(U, W, np, o.partials, blockIdx.x, UX);
	last_block_sum(o.ticket, o.partials, gridDim.x, 4, o.scalars);
}

// Verlet-skin build (only in the steps for which *flag == step, right after the rebinning on the
// skin grid g): every molecule's candidates within rc + skin (rl2, the exact double test of the
// pair kernel with the larger radius) as codes j << 5 | image in the scan order of the pair
// kernel, column k of molecule i at k * n + i; count -1 when more than cap were found (the pair
// kernel then scans the cells); the positions of the build for the displacement check.
__device__ __forceinline__ void rigid_build_one(int64_t i, int64_t n, const double* __restrict__ rx,
                                                const double* __restrict__ ry, const double* __restrict__ rz,
                                                const int32_t* __restrict__ start, const Grid& g, double rl2, int cap,
                                                uint32_t* __restrict__ list, int32_t* __restrict__ count,
                                                double* __restrict__ rref) {
	const double xi = rx[i], yi = ry[i], zi = rz[i];
	rref[i] = xi;
	rref[n + i] = yi;
	rref[2 * n + i] = zi;
	const double r[3] = {xi, yi, zi};
	int cc[3];
	for (int d = 0; d < 3; d++) {
		int c = (int) floor(__ddiv_rn(__dsub_rn(r[d], g.halo_min[d]), g.cell_length[d])) - 1;
		cc[d] = c < 0 ? 0 : (c >= g.nc[d] ? g.nc[d] - 1 : c);
	}
	int cnt = 0;
	for (int dz = -1; dz <= 1; dz++) {
		int z = cc[2] + dz, iz = 1;
		if (z < 0) {
			z += g.nc[2];
			iz = 0;
		} else if (z >= g.nc[2]) {
			z -= g.nc[2];
			iz = 2;
		}
		const double sz = (double) (iz - 1) * g.L[2];
		for (int dy = -1; dy <= 1; dy++) {
			int y = cc[1] + dy, iy = 1;
			if (y < 0) {
				y += g.nc[1];
				iy = 0;
			} else if (y >= g.nc[1]) {
				y -= g.nc[1];
				iy = 2;
			}
			const double sy = (double) (iy - 1) * g.L[1];
			for (int dx = -1; dx <= 1; dx++) {
				int x = cc[0] + dx, ix = 1;
				if (x < 0) {
					x += g.nc[0];
					ix = 0;
				} else if (x >= g.nc[0]) {
					x -= g.nc[0];
					ix = 2;
				}
				const double sx = (double) (ix - 1) * g.L[0];
				const uint32_t img = (uint32_t) (ix + 3 * iy + 9 * iz);
				const bool shifted = img != 13u;
				const int nb = (z * g.nc[1] + y) * g.nc[0] + x;
				const int j0 = start[nb], j1 = start[nb + 1];
				for (int j = j0; j < j1; j++) {
					if (j == i && !shifted) continue;
					const double m0 = __dsub_rn(xi, __dadd_rn(rx[j], sx));
					const double m1 = __dsub_rn(yi, __dadd_rn(ry[j], sy));
					const double m2 = __dsub_rn(zi, __dadd_rn(rz[j], sz));
					const double dd = __dadd_rn(__dadd_rn(__dmul_rn(m0, m0), __dmul_rn(m1, m1)), __dmul_rn(m2, m2));
					if (!(dd < rl2)) continue;
					if (cnt < cap) list[(int64_t) cnt * n + i] = ((uint32_t) j << 5) | img;
					cnt++;
				}
			}
		}
	}
	count[i] = cnt <= cap ? cnt : -1;
}

// (one thread per molecule; the loop covers any grid)
__global__ void __launch_bounds__(kRigidThreads) k_rigid_build(int64_t n, const double* __restrict__ rx,
                                                               const double* __restrict__ ry,
                                                               const double* __restrict__ rz,
                                                               const int32_t* __restrict__ start, Grid g, double rl2,
                                                               const int* flag, int step, int cap,
                                                               uint32_t* __restrict__ list, int32_t* __restrict__ count,
                                                               double* __restrict__ rref,
                                                               unsigned long long* builds) {
	if (*flag != step) return;
	if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(builds, 1ull);
	for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
		rigid_build_one(i, n, rx, ry, rz, start, g, rl2, cap, list, count, rref);
}

struct RigidState {
	double *rx, *ry, *rz, *vx, *vy, *vz;
	const double *fx, *fy, *fz;
	const int32_t* cid;
	const int32_t* uidx;
	double* q;
	double* D;
	const double* M;
};

// Displacement check of the Verlet-skin mode: with rref, a molecule farther than skin/2 from its
// position at the last build (half_skin2 = (skin/2)^2) asks for a build in this step.
struct SkinCheck {
	const double* rref;   // 3 x n, sorted order
	double half_skin2;
	int* flag;
	int step;
};

// Molecule::upd_preF for every molecule
__global__ void __launch_bounds__(kRigidThreads) k_rigid_pre(int64_t n, RigidState s, const RigidParams* __restrict__ P,
                                                             double dt, double vcorr, double Dcorr, SkinCheck sk) {
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int c = s.cid[i];
	const int64_t u = s.uidx ? s.uidx[i] : i;
	const double dt_halve = __dmul_rn(.5, dt);
	const double dtInv2m = __ddiv_rn(dt_halve, P->mass[c]);
	double v0 = __dadd_rn(__dmul_rn(vcorr, s.vx[i]), __dmul_rn(dtInv2m, s.fx[i]));
	double v1 = __dadd_rn(__dmul_rn(vcorr, s.vy[i]), __dmul_rn(dtInv2m, s.fy[i]));
	double v2 = __dadd_rn(__dmul_rn(vcorr, s.vz[i]), __dmul_rn(dtInv2m, s.fz[i]));
	s.vx[i] = v0;
	s.vy[i] = v1;
	s.vz[i] = v2;
	const double x = __dadd_rn(s.rx[i], __dmul_rn(dt, v0));
	const double y = __dadd_rn(s.ry[i], __dmul_rn(dt, v1));
	const double z = __dadd_rn(s.rz[i], __dmul_rn(dt, v2));
	s.rx[i] = x;
	s.ry[i] = y;
	s.rz[i] = z;
	if (sk.rref) {
		const double dx = x - sk.rref[i], dy = y - sk.rref[n + i], dz = z - sk.rref[2 * n + i];
		if (dx * dx + dy * dy + dz * dz > sk.half_skin2) *sk.flag = sk.step;
	}

	const Quat q = load_q(s.q, n, u);
	double D[3] = {s.D[u], s.D[n + u], s.D[2 * n + u]};
	const double M[3] = {s.M[u], s.M[n + u], s.M[2 * n + u]};
	double w[3];
	q_rotate(q, D, w);
	for (int d = 0; d < 3; d++) w[d] = __dmul_rn(w[d], P->invI[c][d]);
	Quat qh = q_add(q_scale(q_differentiate(q, w), dt_halve), q);
	qh = q_scale(qh, __ddiv_rn(1., __dsqrt_rn(q_magnitude2(qh))));
	for (int d = 0; d < 3; d++) D[d] = __dadd_rn(__dmul_rn(Dcorr, D[d]), __dmul_rn(dt_halve, M[d]));
	q_rotate(qh, D, w);
	for (int d = 0; d < 3; d++) w[d] = __dmul_rn(w[d], P->invI[c][d]);
	Quat qn = q_add(q, q_scale(q_differentiate(qh, w), dt));
	qn = q_scale(qn, __ddiv_rn(1., __dsqrt_rn(q_magnitude2(qn))));
	store_q(s.q, n, u, qn);
	s.D[u] = D[0];
	s.D[n + u] = D[1];
	s.D[2 * n + u] = D[2];
}

// Molecule::upd_postF for every molecule; sums m v^2 and I w^2 into scalars[0..1]. With a record
// pointer the last block also writes the step record {Upot, virial, sum m v^2, sum I w^2, pairs}
// from the pair sums in pair_scalars.
__global__ void __launch_bounds__(kRigidThreads) k_rigid_post(int64_t n, RigidState s, const RigidParams* __restrict__ P,
                                                              double dt_half, double* partials, unsigned* ticket,
                                                              double* scalars, const double* pair_scalars,
                                                              double* record, int* status) {
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	double mv2 = 0.0, iw2 = 0.0;
	if (i < n) {
		const int c = s.cid[i];
		const int64_t u = s.uidx ? s.uidx[i] : i;
		const double m = P->mass[c];
		const double dtInv2m = __ddiv_rn(dt_half, m);
		const double v0 = __dadd_rn(s.vx[i], __dmul_rn(dtInv2m, s.fx[i]));
		const double v1 = __dadd_rn(s.vy[i], __dmul_rn(dtInv2m, s.fy[i]));
		const double v2 = __dadd_rn(s.vz[i], __dmul_rn(dtInv2m, s.fz[i]));
		s.vx[i] = v0;
		s.vy[i] = v1;
		s.vz[i] = v2;
		const double vv = __dadd_rn(__dadd_rn(__dmul_rn(v0, v0), __dmul_rn(v1, v1)), __dmul_rn(v2, v2));
		mv2 = __dmul_rn(m, vv);
		double D[3];
		for (int d = 0; d < 3; d++) {
			D[d] = __dadd_rn(s.D[d * n + u], __dmul_rn(dt_half, s.M[d * n + u]));
			s.D[d * n + u] = D[d];
		}
		double w[3];
		q_rotate(load_q(s.q, n, u), D, w);
		for (int d = 0; d < 3; d++) {
			w[d] = __dmul_rn(w[d], P->invI[c][d]);
			iw2 = __dadd_rn(iw2, __dmul_rn(__dmul_rn(P->I[c][d], w[d]), w[d]));
		}
		if (!(isfinite(mv2) && isfinite(iw2))) atomicOr(status, kStatusNonFinite);
	}
	block_sum3(mv2, iw2, 0.0, partials);
	if (last_block_sum(ticket, partials, gridDim.x, 2, scalars) && threadIdx.x == 0 && record) {
		record[0] = pair_scalars[0] * 0.5 / 6. + pair_scalars[3] * 0.5;
		record[1] = pair_scalars[1] * 0.5;
		record[2] = scalars[0];
		record[3] = scalars[1];
		record[4] = pair_scalars[2] * 0.5;
	}
}

// The closing kicks of a step (k_rigid_post, its sums and record) and the opening kicks, drift and
// rotation of the next (k_rigid_pre with vcorr = Dcorr = 1) in one pass over the molecules: the same
// operations in the same order as the two kernels, the intermediate v, D and w kept in registers.
__global__ void __launch_bounds__(kRigidThreads) k_rigid_post_pre(int64_t n, RigidState s,
                                                                  const RigidParams* __restrict__ P, double dt,
                                                                  double* partials, unsigned* ticket, double* scalars,
                                                                  const double* pair_scalars, double* record,
                                                                  int* status, SkinCheck sk) {
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	double mv2 = 0.0, iw2 = 0.0;
	if (i < n) {
		const int c = s.cid[i];
		const int64_t u = s.uidx ? s.uidx[i] : i;
		const double m = P->mass[c];
		const double dt_half = __dmul_rn(.5, dt);
		const double dtInv2m = __ddiv_rn(dt_half, m);
		const double f0 = s.fx[i], f1 = s.fy[i], f2 = s.fz[i];
		// Molecule::upd_postF
		double v0 = __dadd_rn(s.vx[i], __dmul_rn(dtInv2m, f0));
		double v1 = __dadd_rn(s.vy[i], __dmul_rn(dtInv2m, f1));
		double v2 = __dadd_rn(s.vz[i], __dmul_rn(dtInv2m, f2));
		const double vv = __dadd_rn(__dadd_rn(__dmul_rn(v0, v0), __dmul_rn(v1, v1)), __dmul_rn(v2, v2));
		mv2 = __dmul_rn(m, vv);
		const double M[3] = {s.M[u], s.M[n + u], s.M[2 * n + u]};
		double D[3];
		for (int d = 0; d < 3; d++) D[d] = __dadd_rn(s.D[d * n + u], __dmul_rn(dt_half, M[d]));
		const Quat q = load_q(s.q, n, u);
		double w[3];
		q_rotate(q, D, w);
		for (int d = 0; d < 3; d++) {
			w[d] = __dmul_rn(w[d], P->invI[c][d]);
			iw2 = __dadd_rn(iw2, __dmul_rn(__dmul_rn(P->I[c][d], w[d]), w[d]));
		}
		if (!(isfinite(mv2) && isfinite(iw2))) atomicOr(status, kStatusNonFinite);
		// Molecule::upd_preF of the next step
		v0 = __dadd_rn(__dmul_rn(1.0, v0), __dmul_rn(dtInv2m, f0));
		v1 = __dadd_rn(__dmul_rn(1.0, v1), __dmul_rn(dtInv2m, f1));
		v2 = __dadd_rn(__dmul_rn(1.0, v2), __dmul_rn(dtInv2m, f2));
		s.vx[i] = v0;
		s.vy[i] = v1;
		s.vz[i] = v2;
		const double x = __dadd_rn(s.rx[i], __dmul_rn(dt, v0));
		const double y = __dadd_rn(s.ry[i], __dmul_rn(dt, v1));
		const double z = __dadd_rn(s.rz[i], __dmul_rn(dt, v2));
		s.rx[i] = x;
		s.ry[i] = y;
		s.rz[i] = z;
		if (sk.rref) {
			const double dx = x - sk.rref[i], dy = y - sk.rref[n + i], dz = z - sk.rref[2 * n + i];
			if (dx * dx + dy * dy + dz * dz > sk.half_skin2) *sk.flag = sk.step;
		}
		Quat qh = q_add(q_scale(q_differentiate(q, w), dt_half), q);
		qh = q_scale(qh, __ddiv_rn(1., __dsqrt_rn(q_magnitude2(qh))));
		for (int d = 0; d < 3; d++) D[d] = __dadd_rn(__dmul_rn(1.0, D[d]), __dmul_rn(dt_half, M[d]));
		q_rotate(qh, D, w);
		for (int d = 0; d < 3; d++) w[d] = __dmul_rn(w[d], P->invI[c][d]);
		Quat qn = q_add(q, q_scale(q_differentiate(qh, w), dt));
		qn = q_scale(qn, __ddiv_rn(1., __dsqrt_rn(q_magnitude2(qn))));
		store_q(s.q, n, u, qn);
		s.D[u] = D[0];
		s.D[n + u] = D[1];
		s.D[2 * n + u] = D[2];
	}
	block_sum3(mv2, iw2, 0.0, partials);
	if (last_block_sum(ticket, partials, gridDim.x, 2, scalars) && threadIdx.x == 0 && record) {
		record[0] = pair_scalars[0] * 0.5 / 6. + pair_scalars[3] * 0.5;
		record[1] = pair_scalars[1] * 0.5;
		record[2] = scalars[0];
		record[3] = scalars[1];
		record[4] = pair_scalars[2] * 0.5;
	}
}

template <typename T>
__global__ void k_gather_soa(int64_t n, int k, const T* __restrict__ src, T* __restrict__ dst) {
	// (k, n) component-major -> (n, k) row-major
	const int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n * k) return;
	const int64_t i = t / k, d = t % k;
	dst[t] = src[d * n + i];
}

template <typename T>
__global__ void k_scatter_soa(int64_t n, int k, const T* __restrict__ src, T* __restrict__ dst) {
	// (n, k) row-major -> (k, n) component-major
	const int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n * k) return;
	const int64_t i = t / k, d = t % k;
	dst[d * n + i] = src[t];
}

// The skin mode keeps q, D and M in the sorted order of the particle arrays (kRigidPlanes planes of
// n doubles: q 4, D 3, M 3), so that the per-step kernels read them coalesced; the caller's order
// (index uidx of the sorted arrays) is restored when a run ends.
constexpr int kRigidPlanes = 10;

// caller order -> sorted order (to_sorted) or back, plane by plane, for the k planes at src / dst
__global__ void k_state_map(int64_t n, int k, const int32_t* __restrict__ uidx, const double* __restrict__ src,
                            double* __restrict__ dst, bool to_sorted) {
	const int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n * k) return;
	const int64_t d = t / n, i = t % n, u = uidx[i];
	if (to_sorted)
		dst[d * n + i] = src[d * n + u];
	else
		dst[d * n + u] = src[d * n + i];
}

}  // namespace
}  // namespace mdgpu

using namespace mdgpu;

struct mdgpu_rigid {
	mdgpu_ctx* inner = nullptr;
	RigidParams hp{};
	RigidParams* dp = nullptr;
	double* q = nullptr;        // 4 x cap, caller order
	double* D = nullptr;        // 3 x cap
	double* M = nullptr;        // 3 x cap
	double* ds = nullptr;       // 3 x ns_max x cap, sorted order
	float* dsf = nullptr;       // the same in float (mixed form)
	double* es = nullptr;       // rotated orientations of dipoles and quadrupoles, as ds
	float4* rec = nullptr;      // 64-byte partner records of the mixed two-centre variants, sorted order
	double* ss = nullptr;       // the skin mode's q, D, M in sorted order (kRigidPlanes x cap), then as much scratch
	// the components as given (mdgpu_rigid_set_polarities rebuilds the site tables from them)
	int ncomp = 0;
	std::vector<int32_t> nlj_in, nq_in;
	std::vector<mdgpu_site> sites_in;
	std::vector<mdgpu_charge> charges_in;
	std::vector<double> inertia_in, mix_in;
	double* stage = nullptr;    // 4 x cap host <-> device staging
	double* partials = nullptr; // per-block reduction partials (4 doubles per block of the pair kernel)
	double* scal = nullptr;     // [0..2] pair sums, [3..4] kinetic sums
	double* steps = nullptr;    // 5 doubles per step of mdgpu_rigid_run
	int64_t steps_cap = 0;
	unsigned* tickets = nullptr;
	double* h_scal = nullptr;
	int64_t cap = 0;
	// Verlet-skin mode of mdgpu_rigid_run (skin > 0)
	double skin = 0.0;
	int list_cap_req = 0;        // entries per molecule asked for (0: from the densest cell)
	Grid gs{};                   // the skin grid of the loaded positions
	bool gs_valid = false;
	uint32_t* list = nullptr;    // list_cap x list_n codes
	int32_t* list_count = nullptr;
	double* rref = nullptr;      // 3 x list_n positions of the last build
	int list_cap = 0;
	int64_t list_n = 0;
	bool lists_valid = false;    // the sort order has not changed since the lists were built
};

namespace {

Context* ctx_of(mdgpu_rigid* h) { return &h->inner->c; }

#define RG_CUDA(call)                                                       \
	do {                                                                    \
		cudaError_t e_ = (call);                                            \
		if (e_ != cudaSuccess) return set_cuda_error(c, e_, #call);        \
	} while (0)

// Forces of the current positions: on the container's cells, or in the skin mode (skin) from the
// lists on the skin grid.
int launch_rigid_forces(mdgpu_rigid* h, bool skin = false) {
	Context* c = ctx_of(h);
	const int64_t n = c->n;
	const Grid& grid = skin ? h->gs : c->g;
	const RigidLists vl{skin ? h->list : nullptr, skin ? h->list_count : nullptr};
	const unsigned nb = (unsigned) nblocks(n);
	const unsigned nbp = (unsigned) nblocks(n * kRigidLanes);
	prof_begin(c, 1);
	const bool mixed = c->precision == MDGPU_MIXED;
	const int ns = h->hp.ns_max;
	bool charged = false;   // any point polarity: the kernel variant with the polarity blocks
	for (int k = 0; k < h->hp.nc; k++) charged |= h->hp.nsites[k] > h->hp.nlj[k];
	const bool records = mixed && ns <= 2 && !charged && !h->hp.oriented;
	const int32_t* qmap = skin ? nullptr : c->p.uidx;   // the skin mode's q and M are in sorted order
	double* const qsrc = skin ? h->ss : h->q;
	double* const Mdst = skin ? h->ss + 7 * n : h->M;
	k_rigid_sites<<<nb, kRigidThreads, 0, c->stream>>>(n, qmap, c->p.cid, qsrc, h->dp, h->ds,
	                                                   mixed ? h->dsf : nullptr, h->hp.oriented ? h->es : nullptr,
	                                                   c->p.rx, c->p.ry, c->p.rz, records ? h->rec : nullptr);
	RigidOut o{c->p.fx, c->p.fy, c->p.fz, Mdst, h->partials, h->tickets, h->scal, c->status};
#define RG_PAIRS_Q(MX, NSV, QV)                                                                               \
	k_rigid_pairs<MX, NSV, QV><<<nbp, kRigidThreads, 0, c->stream>>>(                                         \
	    n, c->p.rx, c->p.ry, c->p.rz, c->p.cid, qmap, c->cell_start, grid, h->dp, h->ds, h->dsf, h->es, o, vl, h->rec)
#define RG_PAIRS(MX, NSV) \
	(h->hp.oriented ? RG_PAIRS_Q(MX, NSV, 2) : (charged ? RG_PAIRS_Q(MX, NSV, 1) : RG_PAIRS_Q(MX, NSV, 0)))
	if (ns <= 1)
		mixed ? RG_PAIRS(true, 1) : RG_PAIRS(false, 1);
	else if (ns == 2)
		mixed ? RG_PAIRS(true, 2) : RG_PAIRS(false, 2);
	else if (ns == 3)
		mixed ? RG_PAIRS(true, 3) : RG_PAIRS(false, 3);
	else if (ns == 4)
		mixed ? RG_PAIRS(true, 4) : RG_PAIRS(false, 4);
	else
		mixed ? RG_PAIRS(true, kMaxSites) : RG_PAIRS(false, kMaxSites);
#undef RG_PAIRS
#undef RG_PAIRS_Q
	prof_end(c, 1, 2);
	RG_CUDA(cudaGetLastError());
	return MDGPU_OK;
}

// The kernels' view of the state: q, D, M in the caller's order (index uidx), or in the skin mode
// the sorted copies (no index map).
RigidState state_of(mdgpu_rigid* h, bool skin = false) {
	Context* c = ctx_of(h);
	const int64_t n = c->n;
	if (skin)
		return RigidState{c->p.rx, c->p.ry, c->p.rz, c->p.vx, c->p.vy, c->p.vz, c->p.fx, c->p.fy, c->p.fz,
		                  c->p.cid, nullptr, h->ss, h->ss + 4 * n, h->ss + 7 * n};
	return RigidState{c->p.rx, c->p.ry, c->p.rz, c->p.vx, c->p.vy, c->p.vz, c->p.fx, c->p.fy, c->p.fz,
	                  c->p.cid, c->p.uidx, h->q, h->D, h->M};
}

// Copies q, D, M between the caller's order and the sorted copies of the skin mode.
int rigid_state_map(mdgpu_rigid* h, bool to_sorted) {
	Context* c = ctx_of(h);
	const int64_t n = c->n;
	struct {
		double* caller;
		int64_t off;
		int k;
	} sets[3] = {{h->q, 0, 4}, {h->D, 4 * n, 3}, {h->M, 7 * n, 3}};
	for (auto& st : sets) {
		double* sorted = h->ss + st.off;
		k_state_map<<<(unsigned) nblocks(n * st.k), kRigidThreads, 0, c->stream>>>(
		    n, st.k, c->p.uidx, to_sorted ? st.caller : sorted, to_sorted ? sorted : st.caller, to_sorted);
	}
	count_launches(c, 3);
	RG_CUDA(cudaGetLastError());
	return MDGPU_OK;
}

int launch_rigid_pre(mdgpu_rigid* h, double dt, double vcorr, double Dcorr, bool skin_check = false) {
	Context* c = ctx_of(h);
	prof_begin(c, 2);
	const double hs = 0.5 * h->skin;
	const SkinCheck sk{skin_check ? h->rref : nullptr, hs * hs, c->rebuild, c->step_id};
	k_rigid_pre<<<(unsigned) nblocks(c->n), kRigidThreads, 0, c->stream>>>(c->n, state_of(h, skin_check), h->dp, dt,
	                                                                       vcorr, Dcorr, sk);
	prof_end(c, 2, 1);
	RG_CUDA(cudaGetLastError());
	return MDGPU_OK;
}

// The closing kicks of the step (record) and the opening kicks and drift of the next, one launch.
int launch_rigid_post_pre(mdgpu_rigid* h, double dt, double* record, bool skin) {
	Context* c = ctx_of(h);
	prof_begin(c, 2);
	const double hs = 0.5 * h->skin;
	const SkinCheck sk{skin ? h->rref : nullptr, hs * hs, c->rebuild, c->step_id};
	k_rigid_post_pre<<<(unsigned) nblocks(c->n), kRigidThreads, 0, c->stream>>>(
	    c->n, state_of(h, skin), h->dp, dt, h->partials, h->tickets + 1, h->scal + 4, h->scal, record, c->status, sk);
	prof_end(c, 2, 1);
	RG_CUDA(cudaGetLastError());
	return MDGPU_OK;
}

// Buffers and grid of the skin mode for the loaded molecules.
int rigid_skin_prepare(mdgpu_rigid* h) {
	Context* c = ctx_of(h);
	const int64_t n = c->n;
	if (!h->gs_valid) {
		// cells of edge rc + skin: the build scans the 27 cells around each molecule, so unlike the
		// single-centre bricks it gains nothing from larger cells
		std::string err;
		Grid gs{};
		const double length[3] = {c->g.L[0], c->g.L[1], c->g.L[2]};
		const int st = setup_grid(length, c->rc + h->skin, 1.0, gs, err);
		if (st) return set_error(c, st, "cutoff + skin: " + err);
		if (gs.ncells > c->g.ncells) return set_error(c, MDGPU_ERR_ARG, "the skin grid has more cells than the box");
		h->gs = gs;
		h->gs_valid = true;
		h->lists_valid = false;
	}
	int cap = h->list_cap_req;
	if (cap <= 0) {
		// 1.25 x the partners within rc + skin at the densest cell's density, and a margin
		const double rl = c->rc + h->skin;
		const double vol = c->g.cell_length[0] * c->g.cell_length[1] * c->g.cell_length[2];
		const double rho = (c->max_occ > 0 ? c->max_occ : 1) / vol;
		cap = (int) std::ceil(1.25 * 4.18879020478639 * rl * rl * rl * rho) + 16;
	}
	if (h->list_n != n || h->list_cap != cap) {
		cudaFree(h->list);
		cudaFree(h->list_count);
		cudaFree(h->rref);
		h->list = nullptr;
		h->list_count = nullptr;
		h->rref = nullptr;
		h->list_n = 0;
		RG_CUDA(cudaMalloc(&h->list, sizeof(uint32_t) * (size_t) cap * n));
		RG_CUDA(cudaMalloc(&h->list_count, sizeof(int32_t) * n));
		RG_CUDA(cudaMalloc(&h->rref, sizeof(double) * 3 * n));
		h->list_n = n;
		h->list_cap = cap;
		h->lists_valid = false;
	}
	return rebuild_prepare(c);
}

// The build step's rebinning on the skin grid and list build; both return at once unless the
// displacement check (or an invalid list) asked for a build in this step.
int launch_rigid_build(mdgpu_rigid* h) {
	Context* c = ctx_of(h);
	const int64_t n = c->n;
	// the sorted q, D, M move with the molecules
	RG_CUDA(launch_rebuild(c, h->gs, h->ss, h->ss + kRigidPlanes * n, kRigidPlanes));
	prof_begin(c, 0);
	const double rl = c->rc + h->skin;
	k_rigid_build<<<(unsigned) nblocks(n), kRigidThreads, 0, c->stream>>>(
	    c->n, c->p.rx, c->p.ry, c->p.rz, c->cell_start, h->gs, rl * rl, c->rebuild, c->step_id, h->list_cap, h->list,
	    h->list_count, h->rref, c->builds);
	prof_end(c, 0, 1);
	RG_CUDA(cudaGetLastError());
	return MDGPU_OK;
}

int launch_rigid_post(mdgpu_rigid* h, double dt_half, double* record, bool skin = false) {
	Context* c = ctx_of(h);
	prof_begin(c, 2);
	k_rigid_post<<<(unsigned) nblocks(c->n), kRigidThreads, 0, c->stream>>>(
	    c->n, state_of(h, skin), h->dp, dt_half, h->partials, h->tickets + 1, h->scal + 4, h->scal, record, c->status);
	prof_end(c, 2, 1);
	RG_CUDA(cudaGetLastError());
	return MDGPU_OK;
}

// Site tables from the components (Comp2Param::initialize, Component::addLJcenter/addCharge/
// addDipole/addQuadrupole): per component its LJ centres (nlj[k], listed one component after another
// in `sites`), then its charges (ncharges[k] in `charges`), dipoles and quadrupoles (any of these
// lists may be NULL for none). eps_rf: the reaction field's permittivity (epsilonRF).
int setup_rigid(Context* c, int ncomp, const int32_t* nlj, const mdgpu_site* sites, const int32_t* ncharges,
                const mdgpu_charge* charges, const int32_t* ndipoles, const mdgpu_oriented* dipoles,
                const int32_t* nquadrupoles, const mdgpu_oriented* quadrupoles, double eps_rf, const double* inertia,
                const double* mix, double rc, double rc_lj, RigidParams& P) {
	P = RigidParams{};
	P.nc = ncomp;
	P.rc2 = rc * rc;
	P.rclj2 = rc_lj * rc_lj;
	P.eps_rf_inv_rc3 = 2. * (eps_rf - 1.) / ((rc * rc * rc) * (2. * eps_rf + 1.));   // Comp2Param.cpp:178
	int total = 0;
	std::vector<int> lj_off(ncomp), q_off(ncomp), d_off(ncomp), qq_off(ncomp), nq(ncomp), nd(ncomp), nqq(ncomp);
	int lo = 0, qo = 0, dof = 0, qqo = 0;
	for (int k = 0; k < ncomp; k++) {
		nq[k] = ncharges ? ncharges[k] : 0;
		nd[k] = ndipoles ? ndipoles[k] : 0;
		nqq[k] = nquadrupoles ? nquadrupoles[k] : 0;
		if (nlj[k] < 1 || nq[k] < 0 || nd[k] < 0 || nqq[k] < 0 || nlj[k] + nq[k] + nd[k] + nqq[k] > kMaxSites)
			return set_error(c, MDGPU_ERR_ARG, "each component needs at least one LJ centre and at most " +
			                                       std::to_string(kMaxSites) + " sites");
		if ((nq[k] > 0 && !charges) || (nd[k] > 0 && !dipoles) || (nqq[k] > 0 && !quadrupoles))
			return set_error(c, MDGPU_ERR_ARG, "point polarities missing");
		P.nlj[k] = nlj[k];
		P.nsites[k] = nlj[k] + nq[k] + nd[k] + nqq[k];
		P.base[k] = total;
		total += P.nsites[k];
		P.ns_max = std::max(P.ns_max, P.nsites[k]);
		lj_off[k] = lo;
		q_off[k] = qo;
		d_off[k] = dof;
		qq_off[k] = qqo;
		lo += nlj[k];
		qo += nq[k];
		dof += nd[k];
		qqo += nqq[k];
		if (nd[k] + nqq[k] > 0) P.oriented = 1;
	}
	if (total > kMaxSiteTotal)
		return set_error(c, MDGPU_ERR_ARG, "at most " + std::to_string(kMaxSiteTotal) + " sites in all components");
	P.nsite_total = total;
	std::vector<double> shift(total, 0.0);
	for (int k = 0; k < ncomp; k++) {
		double m = 0.0, I[3] = {0.0, 0.0, 0.0};
		auto add_mass = [&](const double r[3], double mass) {
			const double x = r[0], y = r[1], z = r[2];
			m += mass;
			I[0] += mass * (y * y + z * z);
			I[1] += mass * (x * x + z * z);
			I[2] += mass * (x * x + y * y);
		};
		const int b = P.base[k];
		for (int s = 0; s < nlj[k]; s++) {
			const mdgpu_site& t = sites[lj_off[k] + s];
			if (!(t.mass > 0.0) || !(t.sigma > 0.0) || !(t.eps >= 0.0))
				return set_error(c, MDGPU_ERR_ARG, "LJ centre with non-positive mass or sigma, or negative eps");
			for (int d = 0; d < 3; d++) P.site[b + s][d] = t.r[d];
			P.type[b + s] = 0;
			add_mass(t.r, t.mass);
			if (t.do_shift) {   // Component::addLJcenter, with the centre's cutoff = LJCutoffRadius
				const double sigperrc2 = t.sigma * t.sigma / (rc_lj * rc_lj);
				const double sigperrc6 = sigperrc2 * sigperrc2 * sigperrc2;
				shift[b + s] = 24.0 * t.eps * (sigperrc6 - sigperrc6 * sigperrc6);
			}
		}
		int s = nlj[k];
		for (int t = 0; t < nq[k]; t++, s++) {
			const mdgpu_charge& x = charges[q_off[k] + t];
			if (!(x.mass >= 0.0)) return set_error(c, MDGPU_ERR_ARG, "charge with negative mass");
			for (int d = 0; d < 3; d++) P.site[b + s][d] = x.r[d];
			P.charge[b + s] = x.q;
			P.strength[b + s] = x.q;
			P.type[b + s] = 1;
			add_mass(x.r, x.mass);
		}
		for (int kind = 2; kind <= 3; kind++) {   // dipoles, then quadrupoles (massless)
			const int cnt = kind == 2 ? nd[k] : nqq[k];
			const mdgpu_oriented* list = kind == 2 ? dipoles + (nd[k] ? d_off[k] : 0) : quadrupoles + (nqq[k] ? qq_off[k] : 0);
			for (int t = 0; t < cnt; t++, s++) {
				for (int d = 0; d < 3; d++) {
					P.site[b + s][d] = list[t].r[d];
					P.e_body[b + s][d] = list[t].e[d];
				}
				P.strength[b + s] = list[t].strength;
				P.type[b + s] = kind;
			}
		}
		P.mass[k] = m;
		for (int d = 0; d < 3; d++) {
			if (inertia && inertia[3 * k + d] > 0.0) I[d] = inertia[3 * k + d];   // InputOldstyle.cpp:188-195
			P.I[k][d] = I[d];
			P.invI[k][d] = I[d] != 0.0 ? 1.0 / I[d] : 0.0;                           // Molecule.cpp:342-350
		}
	}
	int mixpos = 0;
	for (int ci = 0; ci < ncomp; ci++) {
		for (int a = 0; a < nlj[ci]; a++) {
			const mdgpu_site& A = sites[lj_off[ci] + a];
			for (int b = 0; b < nlj[ci]; b++) {
				const mdgpu_site& B = sites[lj_off[ci] + b];
				const int k = (P.base[ci] + a) * kMaxSiteTotal + P.base[ci] + b;
				double sigma2 = .5 * (A.sigma + B.sigma);
				sigma2 *= sigma2;
				P.eps24[k] = 24. * std::sqrt(A.eps * B.eps);
				P.sig2[k] = sigma2;
				P.shift6[k] = shift[P.base[ci] + a];
			}
		}
		for (int cj = ci + 1; cj < ncomp; cj++) {
			const double xi = mix ? mix[2 * mixpos] : 1.0, eta = mix ? mix[2 * mixpos + 1] : 1.0;
			mixpos++;
			for (int a = 0; a < nlj[ci]; a++) {
				const mdgpu_site& A = sites[lj_off[ci] + a];
				for (int b = 0; b < nlj[cj]; b++) {
					const mdgpu_site& B = sites[lj_off[cj] + b];
					const double epsilon24 = 24. * xi * std::sqrt(A.eps * B.eps);
					double sigma2 = eta * .5 * (A.sigma + B.sigma);
					sigma2 *= sigma2;
					const double sigperrc2 = sigma2 / (rc_lj * rc_lj);
					const double sigperrc6 = sigperrc2 * sigperrc2 * sigperrc2;
					const double shift6combined = epsilon24 * (sigperrc6 - sigperrc6 * sigperrc6);
					const int kij = (P.base[ci] + a) * kMaxSiteTotal + P.base[cj] + b;
					const int kji = (P.base[cj] + b) * kMaxSiteTotal + P.base[ci] + a;
					P.eps24[kij] = P.eps24[kji] = epsilon24;
					P.sig2[kij] = P.sig2[kji] = sigma2;
					P.shift6[kij] = P.shift6[kji] = shift6combined;
				}
			}
		}
	}
	return MDGPU_OK;
}

int ensure_capacity(mdgpu_rigid* h, int64_t n) {
	Context* c = ctx_of(h);
	if (n <= h->cap) return MDGPU_OK;
	cudaFree(h->q);
	cudaFree(h->D);
	cudaFree(h->M);
	cudaFree(h->ds);
	cudaFree(h->dsf);
	cudaFree(h->es);
	cudaFree(h->rec);
	cudaFree(h->ss);
	cudaFree(h->stage);
	cudaFree(h->partials);
	h->q = h->D = h->M = h->ds = h->stage = h->partials = h->es = h->ss = nullptr;
	h->rec = nullptr;
	h->dsf = nullptr;
	h->cap = 0;
	RG_CUDA(cudaMalloc(&h->q, sizeof(double) * 4 * n));
	RG_CUDA(cudaMalloc(&h->D, sizeof(double) * 3 * n));
	RG_CUDA(cudaMalloc(&h->M, sizeof(double) * 3 * n));
	RG_CUDA(cudaMalloc(&h->ds, sizeof(double) * 3 * std::max(1, h->hp.ns_max) * n));
	RG_CUDA(cudaMalloc(&h->dsf, sizeof(float) * 3 * std::max(1, h->hp.ns_max) * n));
	RG_CUDA(cudaMalloc(&h->es, sizeof(double) * 3 * std::max(1, h->hp.ns_max) * n));
	RG_CUDA(cudaMalloc(&h->rec, sizeof(float4) * kRecFloat4 * n));
	RG_CUDA(cudaMalloc(&h->ss, sizeof(double) * 2 * kRigidPlanes * n));
	RG_CUDA(cudaMalloc(&h->stage, sizeof(double) * 4 * n));
	RG_CUDA(cudaMalloc(&h->partials, sizeof(double) * 4 * nblocks(n * kRigidLanes)));
	h->cap = n;
	return MDGPU_OK;
}

}  // namespace

extern "C" {

int mdgpu_rigid_create(mdgpu_rigid** out, const double length[3], double cutoff, double lj_cutoff,
                       double cells_in_cutoff, int ncomp, const int32_t* nsites, const mdgpu_site* sites,
                       const int32_t* ncharges, const mdgpu_charge* charges, const double* inertia, const double* mix,
                       int precision, int device) {
	if (!out) return MDGPU_ERR_ARG;
	*out = nullptr;
	if (ncomp < 1 || ncomp > kMaxSpecies || !nsites || !sites) return MDGPU_ERR_ARG;
	// the single-box context holds the molecule centres; its component table carries each component's
	// total mass (the LJ table of the single-centre kernels is not used here)
	std::vector<mdgpu_component> comps(ncomp);
	int base = 0, qbase = 0;
	for (int k = 0; k < ncomp; k++) {
		const int nq = ncharges ? ncharges[k] : 0;
		if (nsites[k] < 1 || nq < 0 || nsites[k] + nq > kMaxSites || (nq > 0 && !charges)) return MDGPU_ERR_ARG;
		double m = 0.0;
		for (int s = 0; s < nsites[k]; s++) m += sites[base + s].mass;
		for (int s = 0; s < nq; s++) m += charges[qbase + s].mass;
		comps[k] = mdgpu_component{sites[base].eps > 0 ? sites[base].eps : 1.0,
		                           sites[base].sigma > 0 ? sites[base].sigma : 1.0, m > 0 ? m : 1.0, 0};
		base += nsites[k];
		qbase += nq;
	}
	mdgpu_ctx* inner = nullptr;
	int st = mdgpu_create(&inner, length, cutoff, lj_cutoff, cells_in_cutoff, ncomp, comps.data(), mix, precision, device);
	if (st) {
		if (inner) mdgpu_destroy(inner);
		return st;
	}
	mdgpu_rigid* h = new mdgpu_rigid();
	h->inner = inner;
	Context* c = ctx_of(h);
	h->ncomp = ncomp;
	h->nlj_in.assign(nsites, nsites + ncomp);
	h->nq_in.assign(ncomp, 0);
	if (ncharges) h->nq_in.assign(ncharges, ncharges + ncomp);
	h->sites_in.assign(sites, sites + base);
	if (charges && qbase > 0) h->charges_in.assign(charges, charges + qbase);
	if (inertia) h->inertia_in.assign(inertia, inertia + 3 * ncomp);
	if (mix && ncomp > 1) h->mix_in.assign(mix, mix + ncomp * (ncomp - 1));
	st = setup_rigid(c, ncomp, nsites, sites, ncharges, charges, nullptr, nullptr, nullptr, nullptr, 1.0e10, inertia,
	                 mix, c->rc, c->rc_lj, h->hp);
	if (st == MDGPU_OK) {
		cudaError_t e = cudaMalloc(&h->dp, sizeof(RigidParams));
		if (e == cudaSuccess) e = cudaMemcpy(h->dp, &h->hp, sizeof(RigidParams), cudaMemcpyHostToDevice);
		if (e == cudaSuccess) e = cudaMalloc(&h->scal, sizeof(double) * 8);
		if (e == cudaSuccess) e = cudaMemset(h->scal, 0, sizeof(double) * 8);
		if (e == cudaSuccess) e = cudaMalloc(&h->tickets, sizeof(unsigned) * 2);
		if (e == cudaSuccess) e = cudaMemset(h->tickets, 0, sizeof(unsigned) * 2);
		if (e == cudaSuccess) e = cudaMallocHost(&h->h_scal, sizeof(double) * 8);
		if (e != cudaSuccess) st = set_cuda_error(c, e, "mdgpu_rigid_create");
	}
	*out = h;   // returned even on failure so that mdgpu_rigid_last_error can be read
	return st;
}

int mdgpu_rigid_set_polarities(mdgpu_rigid* h, const int32_t* ndipoles, const mdgpu_oriented* dipoles,
                               const int32_t* nquadrupoles, const mdgpu_oriented* quadrupoles, double epsilon_rf) {
	if (!h) return MDGPU_ERR_ARG;
	Context* c = ctx_of(h);
	if (h->cap > 0)
		return set_error(c, MDGPU_ERR_STATE, "point polarities must be set before mdgpu_rigid_set_particles");
	if (!(epsilon_rf > 0.0)) return set_error(c, MDGPU_ERR_ARG, "epsilon_rf must be positive");
	RigidParams P{};
	int st = setup_rigid(c, h->ncomp, h->nlj_in.data(), h->sites_in.data(), h->nq_in.data(),
	                     h->charges_in.empty() ? nullptr : h->charges_in.data(), ndipoles, dipoles, nquadrupoles,
	                     quadrupoles, epsilon_rf, h->inertia_in.empty() ? nullptr : h->inertia_in.data(),
	                     h->mix_in.empty() ? nullptr : h->mix_in.data(), c->rc, c->rc_lj, P);
	if (st) return st;
	h->hp = P;
	RG_CUDA(cudaSetDevice(c->device));
	RG_CUDA(cudaMemcpy(h->dp, &h->hp, sizeof(RigidParams), cudaMemcpyHostToDevice));
	return MDGPU_OK;
}

namespace {

// CutoffCorrections.cpp: radial integrals of the LJ tail beyond rc for centre-centre (TICC),
// centre-site (TICS) and site-site (TISS) pairs, tau the sites' distances from the centres of mass.
double ticc_u(int n, double rc, double sigma2) { return -std::pow(rc, 2 * n + 3) / (std::pow(sigma2, n) * (2 * n + 3)); }
double tics_u(int n, double rc, double sigma2, double tau) {
	return -(std::pow(rc + tau, 2 * n + 3) - std::pow(rc - tau, 2 * n + 3)) * rc /
	           (4 * std::pow(sigma2, n) * tau * (n + 1) * (2 * n + 3)) +
	       (std::pow(rc + tau, 2 * n + 4) - std::pow(rc - tau, 2 * n + 4)) /
	           (4 * std::pow(sigma2, n) * tau * (n + 1) * (2 * n + 3) * (2 * n + 4));
}
double tiss_u(int n, double rc, double sigma2, double tau1, double tau2) {
	const double tp = tau1 + tau2, tm = tau1 - tau2;
	return -(std::pow(rc + tp, 2 * n + 4) - std::pow(rc + tm, 2 * n + 4) - std::pow(rc - tm, 2 * n + 4) +
	         std::pow(rc - tp, 2 * n + 4)) *
	           rc / (8 * std::pow(sigma2, n) * tau1 * tau2 * (n + 1) * (2 * n + 3) * (2 * n + 4)) +
	       (std::pow(rc + tp, 2 * n + 5) - std::pow(rc + tm, 2 * n + 5) - std::pow(rc - tm, 2 * n + 5) +
	        std::pow(rc - tp, 2 * n + 5)) /
	           (8 * std::pow(sigma2, n) * tau1 * tau2 * (n + 1) * (2 * n + 3) * (2 * n + 4) * (2 * n + 5));
}
double ticc_v(int n, double rc, double sigma2) { return 2 * n * ticc_u(n, rc, sigma2); }
double tics_v(int n, double rc, double sigma2, double tau) {
	return -(std::pow(rc + tau, 2 * n + 2) - std::pow(rc - tau, 2 * n + 2)) * rc * rc /
	           (4 * std::pow(sigma2, n) * tau * (n + 1)) -
	       3 * tics_u(n, rc, sigma2, tau);
}
double tiss_v(int n, double rc, double sigma2, double tau1, double tau2) {
	const double tp = tau1 + tau2, tm = tau1 - tau2;
	return -(std::pow(rc + tp, 2 * n + 3) - std::pow(rc + tm, 2 * n + 3) - std::pow(rc - tm, 2 * n + 3) +
	         std::pow(rc - tp, 2 * n + 3)) *
	           rc * rc / (8 * std::pow(sigma2, n) * tau1 * tau2 * (n + 1) * (2 * n + 3)) -
	       3 * tiss_u(n, rc, sigma2, tau1, tau2);
}

}  // namespace

int mdgpu_rigid_far_field_correction(int ncomp, const int32_t* nsites, const mdgpu_site* sites, const int32_t* ncharges,
                                     const mdgpu_charge* charges, const int32_t* ndipoles,
                                     const mdgpu_oriented* dipoles, const double* mix, const int64_t* counts,
                                     const double length[3], double cutoff, double lj_cutoff, double epsilon_rf,
                                     double* upot_corr, double* virial_corr, char* errbuf, int errlen) {
	if (errbuf && errlen > 0) errbuf[0] = '\0';
	auto fail = [&](int code, const std::string& msg) {
		if (errbuf && errlen > 0) snprintf(errbuf, (size_t) errlen, "%s", msg.c_str());
		return code;
	};
	if (ncomp < 1 || ncomp > kMaxSpecies) return fail(MDGPU_ERR_ARG, "ncomp must be in 1..8");
	if (!nsites || !sites || !counts || !length) return fail(MDGPU_ERR_ARG, "null argument");
	if (!(cutoff > 0.0)) return fail(MDGPU_ERR_ARG, "cutoff must be positive");
	if (!(lj_cutoff >= 0.0)) return fail(MDGPU_ERR_ARG, "lj_cutoff must be 0 (= cutoff) or positive");
	for (int d = 0; d < 3; d++)
		if (!(length[d] > 0.0)) return fail(MDGPU_ERR_ARG, "box lengths must be positive");
	for (int i = 0; i < ncomp; i++) {
		if (counts[i] < 0) return fail(MDGPU_ERR_ARG, "molecule counts must not be negative");
		if (ndipoles && ndipoles[i] < 0) return fail(MDGPU_ERR_ARG, "dipole counts must not be negative");
	}
	if (ndipoles && !dipoles) {
		for (int i = 0; i < ncomp; i++)
			if (ndipoles[i] > 0) return fail(MDGPU_ERR_ARG, "dipoles are counted but not given");
	}
	if (ndipoles && dipoles) {
		int off = 0;
		for (int i = 0; i < ncomp; i++)
			for (int s = 0; s < ndipoles[i]; s++, off++) {
				const double* e = dipoles[off].e;
				// the reference divides by |e| (Domain.cpp:596-603): a zero direction has no dipole
				if (!(e[0] * e[0] + e[1] * e[1] + e[2] * e[2] > 0.0))
					return fail(MDGPU_ERR_ARG, "a dipole direction has zero length");
			}
	}
	const double rc_lj = lj_cutoff > 0.0 ? lj_cutoff : cutoff;
	Context c;   // host-only: receives the error text of the table set-up
	RigidParams P;
	int st = setup_rigid(&c, ncomp, nsites, sites, ncharges, charges, nullptr, nullptr, nullptr, nullptr, epsilon_rf,
	                     nullptr, mix, cutoff, rc_lj, P);
	if (st) return fail(st, c.err);
	double upot_lj = 0., virial_lj = 0., self_term = 0.;
	int64_t nmol = 0;
	int lo = 0, qo = 0, dof = 0;
	std::vector<int> lj_off(ncomp);
	for (int i = 0; i < ncomp; ++i) {
		lj_off[i] = lo;
		lo += nsites[i];
	}
	for (int i = 0; i < ncomp; ++i) {
		nmol += counts[i];
		// the molecule's dipole from its charges and dipoles (Domain.cpp:586-609)
		double balance[3] = {0., 0., 0.};
		const int nq = ncharges ? ncharges[i] : 0, nd = ndipoles ? ndipoles[i] : 0;
		for (int s = 0; s < nq; s++)
			for (int d = 0; d < 3; d++) balance[d] += charges[qo + s].q * charges[qo + s].r[d];
		for (int s = 0; s < nd; s++) {
			const mdgpu_oriented& t = dipoles[dof + s];
			double evect = 0;
			for (int d = 0; d < 3; d++) evect += t.e[d] * t.e[d];
			const double norm = 1.0 / std::sqrt(evect);
			for (int d = 0; d < 3; d++) balance[d] += t.strength * t.e[d] * norm;
		}
		qo += nq;
		dof += nd;
		double my2 = 0.0;
		for (int d = 0; d < 3; d++) my2 += balance[d] * balance[d];
		self_term += my2 * (double) counts[i];
		for (int j = 0; j < ncomp; ++j) {
			for (int si = 0; si < nsites[i]; ++si) {
				const double* ri = sites[lj_off[i] + si].r;
				const double tau1 = std::sqrt(ri[0] * ri[0] + ri[1] * ri[1] + ri[2] * ri[2]);
				for (int sj = 0; sj < nsites[j]; ++sj) {
					const double* rj = sites[lj_off[j] + sj].r;
					double tau2 = std::sqrt(rj[0] * rj[0] + rj[1] * rj[1] + rj[2] * rj[2]);
					if (tau1 + tau2 >= rc_lj)   // "rc too small" (Domain.cpp:622-625)
						return fail(MDGPU_ERR_ARG, "LJ cutoff too small: two LJ centres' distances from their centres of "
						                           "mass add up to the cutoff or more");
					const int k = (P.base[i] + si) * kMaxSiteTotal + P.base[j] + sj;
					if (P.shift6[k] != 0.0) continue;   // truncated-shifted pairs have no tail correction
					const double eps24 = P.eps24[k], sig2 = P.sig2[k];
					const double fac = double(counts[i]) * double(counts[j]) * eps24;
					if (tau1 == 0. && tau2 == 0.) {
						upot_lj += fac * (ticc_u(-6, rc_lj, sig2) - ticc_u(-3, rc_lj, sig2));
						virial_lj += fac * (ticc_v(-6, rc_lj, sig2) - ticc_v(-3, rc_lj, sig2));
					} else if (tau1 != 0. && tau2 != 0.) {
						upot_lj += fac * (tiss_u(-6, rc_lj, sig2, tau1, tau2) - tiss_u(-3, rc_lj, sig2, tau1, tau2));
						virial_lj += fac * (tiss_v(-6, rc_lj, sig2, tau1, tau2) - tiss_v(-3, rc_lj, sig2, tau1, tau2));
					} else {
						if (tau2 == 0.) tau2 = tau1;
						upot_lj += fac * (tics_u(-6, rc_lj, sig2, tau2) - tics_u(-3, rc_lj, sig2, tau2));
						virial_lj += fac * (tics_v(-6, rc_lj, sig2, tau2) - tics_v(-3, rc_lj, sig2, tau2));
					}
				}
			}
		}
	}
	if (nmol <= 0) return fail(MDGPU_ERR_ARG, "the box holds no molecules");
	const double rho = double(nmol) / (length[0] * length[1] * length[2]);
	const double fac = M_PI * rho / (3. * double(nmol));
	upot_lj *= fac;
	virial_lj *= -fac;
	const double eps_rf_inv_rc3 = 2. * (epsilon_rf - 1.) / ((cutoff * cutoff * cutoff) * (2. * epsilon_rf + 1.));
	self_term *= -0.5 * eps_rf_inv_rc3;
	if (upot_corr) *upot_corr = upot_lj + self_term;
	if (virial_corr) *virial_corr = virial_lj + 3. * self_term;
	return MDGPU_OK;
}

int mdgpu_rigid_destroy(mdgpu_rigid* h) {
	if (!h) return MDGPU_ERR_ARG;
	if (h->inner) cudaSetDevice(h->inner->c.device);
	cudaFree(h->dp);
	cudaFree(h->q);
	cudaFree(h->D);
	cudaFree(h->M);
	cudaFree(h->ds);
	cudaFree(h->dsf);
	cudaFree(h->es);
	cudaFree(h->rec);
	cudaFree(h->ss);
	cudaFree(h->stage);
	cudaFree(h->partials);
	cudaFree(h->scal);
	cudaFree(h->steps);
	cudaFree(h->tickets);
	cudaFree(h->list);
	cudaFree(h->list_count);
	cudaFree(h->rref);
	if (h->h_scal) cudaFreeHost(h->h_scal);
	int st = h->inner ? mdgpu_destroy(h->inner) : MDGPU_OK;
	delete h;
	return st;
}

const char* mdgpu_rigid_last_error(const mdgpu_rigid* h) {
	return h && h->inner ? h->inner->c.err.c_str() : "null context";
}

int mdgpu_rigid_set_precision(mdgpu_rigid* h, int precision) {
	if (!h) return MDGPU_ERR_ARG;
	return mdgpu_set_precision(h->inner, precision);
}

int mdgpu_rigid_get_inertia(const mdgpu_rigid* h, int32_t comp, double* mass, double I[3]) {
	if (!h || comp < 0 || comp >= h->hp.nc) return MDGPU_ERR_ARG;
	if (mass) *mass = h->hp.mass[comp];
	if (I)
		for (int d = 0; d < 3; d++) I[d] = h->hp.I[comp][d];
	return MDGPU_OK;
}

int mdgpu_rigid_set_particles(mdgpu_rigid* h, int64_t n, const uint64_t* id, const int32_t* cid, const double* r,
                              const double* v, const double* q, const double* D) {
	if (!h) return MDGPU_ERR_ARG;
	Context* c = ctx_of(h);
	if (!q || !D) return set_error(c, MDGPU_ERR_ARG, "q and D are required");
	if (n > (int64_t(1) << 27)) return set_error(c, MDGPU_ERR_ARG, "at most 2^27 rigid molecules");
	int st = mdgpu_set_particles(h->inner, n, id, cid, r, v, nullptr);
	if (st) return st;
	st = ensure_capacity(h, n);
	if (st) return st;
	const unsigned nb4 = (unsigned) nblocks(4 * n), nb3 = (unsigned) nblocks(3 * n);
	RG_CUDA(cudaMemcpyAsync(h->stage, q, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, c->stream));
	k_scatter_soa<double><<<nb4, kRigidThreads, 0, c->stream>>>(n, 4, h->stage, h->q);
	RG_CUDA(cudaStreamSynchronize(c->stream));
	RG_CUDA(cudaMemcpyAsync(h->stage, D, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
	k_scatter_soa<double><<<nb3, kRigidThreads, 0, c->stream>>>(n, 3, h->stage, h->D);
	RG_CUDA(cudaMemsetAsync(h->M, 0, sizeof(double) * 3 * n, c->stream));
	RG_CUDA(cudaGetLastError());
	RG_CUDA(cudaStreamSynchronize(c->stream));
	h->gs_valid = false;   // the skin grid follows the density of the new positions
	h->lists_valid = false;
	return MDGPU_OK;
}

int mdgpu_rigid_get_particles(mdgpu_rigid* h, int64_t n, uint64_t* id, int32_t* cid, double* r, double* v, double* F,
                              double* q, double* D, double* M) {
	if (!h) return MDGPU_ERR_ARG;
	Context* c = ctx_of(h);
	int st = mdgpu_get_particles(h->inner, n, id, cid, r, v, F);
	if (st) return st;
	struct {
		double* out;
		const double* src;
		int k;
	} sets[3] = {{q, h->q, 4}, {D, h->D, 3}, {M, h->M, 3}};
	for (auto& s : sets) {
		if (!s.out) continue;
		k_gather_soa<double><<<(unsigned) nblocks(s.k * n), kRigidThreads, 0, c->stream>>>(n, s.k, s.src, h->stage);
		RG_CUDA(cudaMemcpyAsync(s.out, h->stage, sizeof(double) * s.k * n, cudaMemcpyDeviceToHost, c->stream));
		RG_CUDA(cudaStreamSynchronize(c->stream));
	}
	RG_CUDA(cudaGetLastError());
	return MDGPU_OK;
}

int mdgpu_rigid_update(mdgpu_rigid* h) {
	if (!h) return MDGPU_ERR_ARG;
	h->lists_valid = false;   // the sort order changes
	return mdgpu_update(h->inner);
}

int mdgpu_rigid_traverse_pairs(mdgpu_rigid* h, double* upot, double* virial, double* npairs) {
	if (!h) return MDGPU_ERR_ARG;
	Context* c = ctx_of(h);
	if (!c->cells_valid)
		return set_error(c, MDGPU_ERR_STATE, "cell structure in the container is invalid, call mdgpu_rigid_update first");
	RG_CUDA(cudaSetDevice(c->device));
	int st = launch_rigid_forces(h);
	if (st) return st;
	RG_CUDA(cudaMemcpyAsync(h->h_scal, h->scal, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->stream));
	st = check_device_status(c);
	if (st) return st;
	// ParticlePairs2PotForceAdapter::finish: Upot = Upot6LJ/6 + UpotXpoles (each pair was seen twice)
	if (upot) *upot = h->h_scal[0] * 0.5 / 6. + h->h_scal[3] * 0.5;
	if (virial) *virial = h->h_scal[1] * 0.5;
	if (npairs) *npairs = h->h_scal[2] * 0.5;
	return MDGPU_OK;
}

int mdgpu_rigid_leapfrog_pre(mdgpu_rigid* h, double dt, double vcorr, double Dcorr) {
	if (!h) return MDGPU_ERR_ARG;
	Context* c = ctx_of(h);
	if (c->n == 0) return set_error(c, MDGPU_ERR_STATE, "no molecules loaded");
	RG_CUDA(cudaSetDevice(c->device));
	int st = launch_rigid_pre(h, dt, vcorr, Dcorr);
	c->cells_valid = false;
	h->lists_valid = false;   // moved without the displacement check
	return st;
}

int mdgpu_rigid_leapfrog_post(mdgpu_rigid* h, double dt_half, double* summv2, double* sum_iw2) {
	if (!h) return MDGPU_ERR_ARG;
	Context* c = ctx_of(h);
	if (c->n == 0) return set_error(c, MDGPU_ERR_STATE, "no molecules loaded");
	RG_CUDA(cudaSetDevice(c->device));
	int st = launch_rigid_post(h, dt_half, nullptr);
	if (st) return st;
	RG_CUDA(cudaMemcpyAsync(h->h_scal + 4, h->scal + 4, sizeof(double) * 2, cudaMemcpyDeviceToHost, c->stream));
	st = check_device_status(c);
	if (st) return st;
	if (summv2) *summv2 = h->h_scal[4];
	if (sum_iw2) *sum_iw2 = h->h_scal[5];
	return MDGPU_OK;
}

int mdgpu_rigid_run(mdgpu_rigid* h, int32_t nsteps, double dt, double* per_step) {
	if (!h) return MDGPU_ERR_ARG;
	Context* c = ctx_of(h);
	if (nsteps < 0) return set_error(c, MDGPU_ERR_ARG, "nsteps must be >= 0");
	if (c->n == 0) return set_error(c, MDGPU_ERR_STATE, "no molecules loaded");
	RG_CUDA(cudaSetDevice(c->device));
	if (nsteps > h->steps_cap) {
		cudaFree(h->steps);
		h->steps = nullptr;
		h->steps_cap = 0;
		RG_CUDA(cudaMalloc(&h->steps, sizeof(double) * 5 * nsteps));
		h->steps_cap = nsteps;
	}
	if (h->skin > 0.0 && nsteps > 0) {
		int st = rigid_skin_prepare(h);
		if (!st) st = rigid_state_map(h, true);
		if (st) return st;
	}
	int st = MDGPU_OK;
	for (int32_t k = 0; k < nsteps && !st; k++) {
		// Simulation::simulateStep: upd_preF, update (wrap, bin), upd_cache + traversePairs, upd_postF
		double* record = h->steps + 5 * (int64_t) k;
		if (h->skin > 0.0) {
			// the Verlet-skin step: the rebinning and the list build run only when a molecule moved
			// more than skin/2 since the last build (or the lists do not fit the sort order); the
			// closing kicks of a step and the opening kicks of the next run as one pass
			if (k == 0) {
				c->step_id++;
				if (!h->lists_valid) {
					st = request_build(c);
					h->lists_valid = true;
				}
				if (!st) st = launch_rigid_pre(h, dt, 1.0, 1.0, true);
			}
			if (!st) st = launch_rigid_build(h);
			if (!st) st = launch_rigid_forces(h, true);
			if (!st && k + 1 < nsteps) {
				c->step_id++;   // the next step's displacement check asks for its build
				st = launch_rigid_post_pre(h, dt, record, true);
			} else if (!st) {
				st = launch_rigid_post(h, 0.5 * dt, record, true);
			}
		} else {
			st = launch_rigid_pre(h, dt, 1.0, 1.0);
			if (!st) {
				const cudaError_t e = launch_bin(c, true);
				if (e != cudaSuccess) st = set_cuda_error(c, e, "launch_bin");
			}
			if (!st) st = launch_rigid_forces(h);
			if (!st) st = launch_rigid_post(h, 0.5 * dt, record);
		}
	}
	if (h->skin <= 0.0) {
		c->cells_valid = true;
	} else if (nsteps > 0) {
		c->cells_valid = false;   // the cells are the skin grid's, the positions not wrapped
		const int back = rigid_state_map(h, false);   // q, D, M back in the caller's order
		if (!st) st = back;
	}
	if (st) return st;
	c->lists_valid = false;
	if (per_step && nsteps > 0)
		RG_CUDA(cudaMemcpyAsync(per_step, h->steps, sizeof(double) * 5 * nsteps, cudaMemcpyDeviceToHost, c->stream));
	return check_device_status(c);
}

int mdgpu_rigid_set_skin(mdgpu_rigid* h, double skin, int32_t list_cap) {
	if (!h) return MDGPU_ERR_ARG;
	Context* c = ctx_of(h);
	if (!(skin >= 0.0)) return set_error(c, MDGPU_ERR_ARG, "skin must not be negative");
	if (skin > 0.5 * c->rc) return set_error(c, MDGPU_ERR_ARG, "skin must not exceed half the cutoff");
	if (list_cap < 0 || list_cap > (1 << 16)) return set_error(c, MDGPU_ERR_ARG, "list capacity must be in 0..65536");
	if (skin != h->skin) {
		h->gs_valid = false;
		h->lists_valid = false;
	}
	h->skin = skin;
	h->list_cap_req = list_cap;
	return MDGPU_OK;
}

int mdgpu_rigid_skin_builds(mdgpu_rigid* h, int64_t* builds) {
	if (!h || !builds) return MDGPU_ERR_ARG;
	Context* c = ctx_of(h);
	unsigned long long b = 0;
	if (c->builds) {
		RG_CUDA(cudaSetDevice(c->device));
		RG_CUDA(cudaMemcpyAsync(&b, c->builds, sizeof(b), cudaMemcpyDeviceToHost, c->stream));
		RG_CUDA(cudaStreamSynchronize(c->stream));
	}
	*builds = (int64_t) b;
	return MDGPU_OK;
}

int mdgpu_rigid_get_stream(const mdgpu_rigid* h, void** stream) {
	if (!h || !stream) return MDGPU_ERR_ARG;
	return mdgpu_get_stream(h->inner, stream);
}

int mdgpu_rigid_profile_enable(mdgpu_rigid* h, int enable) {
	if (!h) return MDGPU_ERR_ARG;
	return mdgpu_profile_enable(h->inner, enable);
}

int mdgpu_rigid_profile_read(mdgpu_rigid* h, double times_ms[3], int64_t counts[4], int reset) {
	if (!h) return MDGPU_ERR_ARG;
	return mdgpu_profile_read(h->inner, times_ms, counts, reset);
}

}  // extern "C"
