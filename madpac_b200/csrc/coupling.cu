// Molecule-side operations of MaDPaC's coupled MD step on the device container.
//
// MarDynSimulation::simulateStep (coupling/MarDynSimulation.cpp:61-160; paths relative to the
// reference bundle's mardyn/) interleaves the MD step with the lattice-Boltzmann connector's
// operations on molecules. The molecule-side ones, with the connector's parameters as arguments:
//
//  * mdgpu_reflect_boundary: ReflectingBoundary::applyBoundary (coupling/boundary/
//    ReflectingBoundary.cpp:47-130): each molecule outside the box in dimension i < dim has v_i
//    negated and is moved back inside -- by r + (-r - 2r) at the lower face and r - 2 (r - L) at the
//    upper face, the reference's own arithmetic -- except beyond the stream-out face when the
//    stream-out is on, where it is counted and left where it is. In the coupled step it runs after
//    the drift and before the binning;
//  * mdgpu_force_boundary: the wall force ForceBoundary::applyBoundary (coupling/boundary/
//    ForceBoundary.cpp:52-226) computes for the molecules of the boundary regions (within `border`
//    of a face, FBoundary::getLower/getUpper), ForceBoundary::calcFm's piecewise fit
//    (ForceBoundary.h:56-82) in the same operation order; after the pair forces;
//  * mdgpu_thermostat_*: CellWiseThermostat::applyThermostat (coupling/thermostat/
//    CellWiseThermostat.cpp:46-156) on the connector's coupling-cell grid (DataContainer::
//    calcIndexX, madpac/core/DataContainer.cpp:209-261): every call adds each molecule's velocity to
//    its cell's sums; every `interval` calls the cells' mean velocities (in the directed
//    dimensions), their peculiar kinetic energies and the rescaling v = (v - vc)(1 + gamma (beta - 1))
//    + vc with beta = sqrt(1.5 N_samples / interval T / E_cell); after the closing kick.
//
// Sums over molecules use 64-bit fixed point (velocities and energies in steps of 2^-40), so the
// results do not depend on the order in which atomics land; a per-cell sum of 2^23 or more would
// wrap, which a double sum kept beside it detects (status kStatusRange, an error of the call).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>

#include "md_internal.h"

namespace mdgpu {
namespace {

constexpr int kT = 256;
inline unsigned nblk(int64_t n) { return (unsigned) ((n + kT - 1) / kT); }

constexpr double kVScale = 1099511627776.0;   // 2^40
constexpr double kEScale = 1099511627776.0;   // 2^40

// A fixed-point sum that disagrees with its double shadow by 1 or more has wrapped (a wrap moves it
// by 2^24; the shadow's own rounding is many orders below 1 for sums in range).
__device__ __forceinline__ void check_range(unsigned long long fixed, double scale, double shadow, int* status) {
	if (!(fabs((double) (long long) fixed / scale - shadow) < 1.0)) atomicOr(status, kStatusRange);
}

__global__ void k_reflect(int64_t n, Particles p, Grid g, int dim, int sod, bool so, unsigned long long* nout) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	double* rr[3] = {p.rx, p.ry, p.rz};
	double* vv[3] = {p.vx, p.vy, p.vz};
	double r[3] = {p.rx[s], p.ry[s], p.rz[s]};
	double v[3] = {p.vx[s], p.vy[s], p.vz[s]};
	bool moved = false;
	unsigned out = 0;
	for (int i = 0; i < dim; i++) {
		const bool lower = r[i] < 0.0;
		const bool upper = !lower && r[i] > g.L[i];
		if (upper && i == sod && so) {
			out++;
			continue;
		}
		if (!lower && !upper) continue;
		// v += a with a_i = -2 v_i and 0 elsewhere (Molecule::vadd)
		double a[3] = {0.0, 0.0, 0.0};
		a[i] = __dmul_rn(-2.0, v[i]);
		for (int d = 0; d < 3; d++) v[d] = __dadd_rn(v[d], a[d]);
		const double newpos = lower ? __dsub_rn(-r[i], __dmul_rn(2.0, r[i])) : __dmul_rn(-2.0, __dsub_rn(r[i], g.L[i]));
		r[i] = __dadd_rn(r[i], newpos);   // Molecule::move
		moved = true;
	}
	if (moved)
		for (int d = 0; d < 3; d++) {
			rr[d][s] = r[d];
			vv[d][s] = v[d];
		}
	if (out) atomicAdd(nout, (unsigned long long) out);
}

// ForceBoundary::calcFm, left-to-right products and sums without contraction: c * r_w * r_w is
// (c * r_w) * r_w, as the reference's expression evaluates
__device__ double calc_fm(double r) {
	const double rw = __ddiv_rn(r, 2.95);
	auto term = [&](double c, int k) {
		double x = c;
		for (int j = 0; j < k; j++) x = __dmul_rn(x, rw);
		return x;
	};
	if (rw < 0.2975)
		return __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(10.8007, term(0.860717, 1)), -term(172.468, 2)), term(86.9134, 3)),
		                 -term(140.214, 4));
	if (rw < 0.3475)
		return __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(-3621.30, term(44657.4, 1)), -term(204844.0, 2)),
		                           term(414123.0, 3)),
		                 -term(311674.0, 4));
	if (rw < 0.3975)
		return __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(4331.63, -term(45188.5, 1)), term(176236.0, 2)),
		                           -term(305157.0, 3)),
		                 term(198111.0, 4));
	if (rw < 1.0)
		return __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(-94.4796, term(576.282, 1)), -term(1436.11, 2)),
		                                     term(1804.53, 3)),
		                           -term(1133.47, 4)),
		                 term(283.244, 5));
	return 0.0;
}

__global__ void k_force_boundary(int64_t n, Particles p, Grid g, int dim, double border, int sod, double damping) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const double r[3] = {p.rx[s], p.ry[s], p.rz[s]};
	double* ff[3] = {p.fx, p.fy, p.fz};
	bool inside = true;
	for (int d = 0; d < 3; d++) inside = inside && r[d] >= 0.0 && r[d] < g.L[d];
	if (!inside) return;
	const int nd = dim == 3 ? 3 : 2;
	for (int d = 0; d < nd; d++) {
		double F = ff[d][s];
		bool changed = false;
		if (r[d] < 0.0 + border) {
			F = __dadd_rn(F, __dmul_rn(calc_fm(__dsub_rn(r[d], 0.0)), 1.0));
			changed = true;
		}
		if (r[d] >= __dsub_rn(g.L[d], border)) {
			double f = __dmul_rn(-calc_fm(__dsub_rn(g.L[d], r[d])), 1.0);
			if (sod == d) f = __dmul_rn(f, damping);
			F = __dadd_rn(F, f);
			changed = true;
		}
		if (changed) ff[d][s] = F;
	}
}

struct CellGrid {
	double lower[3], upper[3], cell;
	int size[3], dim;
};

// DataContainer::calcIndexX: the coupling cell of a position, -1 outside the coupling box (also at
// its upper corner, where the reference's index would run past its array)
__device__ int coupling_cell(const CellGrid& c, const double pos[3]) {
	int ip[3] = {0, 0, 0};
	for (int i = 0; i < c.dim; i++) {
		if (!(c.lower[i] <= pos[i] && pos[i] <= c.upper[i])) return -1;
		ip[i] = (int) __ddiv_rn(__dsub_rn(pos[i], c.lower[i]), c.cell);
		if (ip[i] >= c.size[i]) return -1;
	}
	return (ip[0] * c.size[1] + ip[1]) * c.size[2] + ip[2];
}

__global__ void k_th_save(int64_t n, Particles p, CellGrid cg, unsigned long long* vsum, double* shadow) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const double pos[3] = {p.rx[s], p.ry[s], p.rz[s]};
	const int k = coupling_cell(cg, pos);
	if (k < 0) return;
	const double v[3] = {p.vx[s], p.vy[s], p.vz[s]};
	for (int i = 0; i < 3; i++) {
		atomicAdd(vsum + 4 * k + i, (unsigned long long) __double2ll_rn(v[i] * kVScale));
		atomicAdd(shadow + 4 * k + i, v[i]);
	}
	atomicAdd(vsum + 4 * k + 3, 1ull);
}

__global__ void k_th_cells(int ncells, const unsigned long long* vsum, int dx, int dy, int dz, double* vc,
                           unsigned long long* esum, double* shadow, int* status) {
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= ncells) return;
	const double cnt = (double) (long long) vsum[4 * k + 3];
	const int dir[3] = {dx, dy, dz};
	for (int i = 0; i < 3; i++) {
		check_range(vsum[4 * k + i], kVScale, shadow[4 * k + i], status);
		vc[3 * k + i] = dir[i] != 0 ? ((double) (long long) vsum[4 * k + i] / kVScale) / cnt : 0.0;
	}
	esum[k] = 0ull;
	shadow[4 * k + 3] = 0.0;
}

__global__ void k_th_energy(int64_t n, Particles p, CellGrid cg, Species sp, const double* vc, unsigned long long* esum,
                            double* shadow) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const double pos[3] = {p.rx[s], p.ry[s], p.rz[s]};
	const int k = coupling_cell(cg, pos);
	if (k < 0) return;
	const double v[3] = {p.vx[s], p.vy[s], p.vz[s]};
	double e = 0.0;
	for (int i = 0; i < 3; i++) {
		const double t = __dsub_rn(v[i], vc[3 * k + i]);
		e = __dadd_rn(e, __dmul_rn(t, t));
	}
	e = __dmul_rn(e, __dmul_rn(0.5, sp.mass[p.cid[s]]));
	atomicAdd(esum + k, (unsigned long long) __double2ll_rn(e * kEScale));
	atomicAdd(shadow + 4 * k + 3, e);
}

__global__ void k_th_adjust(int64_t n, Particles p, CellGrid cg, const unsigned long long* vsum, const double* vc,
                            const unsigned long long* esum, const double* shadow, int* status, double interval,
                            double T, double gamma) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const double pos[3] = {p.rx[s], p.ry[s], p.rz[s]};
	const int k = coupling_cell(cg, pos);
	if (k < 0) return;
	check_range(esum[k], kEScale, shadow[4 * k + 3], status);
	const double target = __dmul_rn(__ddiv_rn(__dmul_rn(1.5, (double) (long long) vsum[4 * k + 3]), interval), T);
	const double beta = __dsqrt_rn(__ddiv_rn(target, (double) (long long) esum[k] / kEScale));
	const double f = __dadd_rn(1.0, __dmul_rn(gamma, __dsub_rn(beta, 1.0)));
	double* vv[3] = {p.vx, p.vy, p.vz};
	for (int i = 0; i < 3; i++) vv[i][s] = __dadd_rn(__dmul_rn(__dsub_rn(vv[i][s], vc[3 * k + i]), f), vc[3 * k + i]);
}

}  // namespace
}  // namespace mdgpu

using namespace mdgpu;

struct mdgpu_thermostat {
	mdgpu_ctx* ctx;
	int device;
	CellGrid cg;
	int ncells;
	double T, gamma;
	int interval;
	int directed[3];
	unsigned long long* vsum;   // 4 per cell: fixed-point v sums and the sample count
	unsigned long long* esum;   // per cell, fixed point
	double* vc;                 // 3 per cell
	double* shadow;             // 4 per cell: the sums in double, to detect a wrap
};

extern "C" {

int mdgpu_reflect_boundary(mdgpu_ctx* ctx, int32_t dim, int32_t stream_out_dir, int32_t moving_wall, int32_t stream_out,
                           int64_t* streamed_out) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (dim != 2 && dim != 3) return set_error(c, MDGPU_ERR_ARG, "dim must be 2 or 3");
	if (c->skin > 0.0) return set_error(c, MDGPU_ERR_STATE, "the coupling operations need the per-step binning (skin 0)");
	if (c->n == 0) return set_error(c, MDGPU_ERR_STATE, "no molecules loaded");
	cudaError_t e = cudaSetDevice(c->device);
	unsigned long long* d_out = reinterpret_cast<unsigned long long*>(c->scalars + 32);
	if (e == cudaSuccess) e = cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), c->stream);
	// ReflectingBoundary.cpp:33: without a moving wall the stream-out face always lets molecules go
	const bool so = !moving_wall || stream_out;
	if (e == cudaSuccess) {
		k_reflect<<<nblk(c->n), kT, 0, c->stream>>>(c->n, c->p, c->g, dim, stream_out_dir, so, d_out);
		count_launches(c, 1);
		e = cudaGetLastError();
	}
	unsigned long long h = 0;
	if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_out, sizeof(h), cudaMemcpyDeviceToHost, c->stream);
	if (e != cudaSuccess) return set_cuda_error(c, e, "mdgpu_reflect_boundary");
	const int st = check_device_status(c);
	if (st) return st;
	c->cells_valid = false;   // positions changed: bin again (LinkedCells::update) before the forces
	if (streamed_out) *streamed_out = (int64_t) h;
	return MDGPU_OK;
}

int mdgpu_force_boundary(mdgpu_ctx* ctx, int32_t dim, double border, int32_t stream_out_dir, double stream_damping) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (dim != 2 && dim != 3) return set_error(c, MDGPU_ERR_ARG, "dim must be 2 or 3");
	if (!(border >= 0.0)) return set_error(c, MDGPU_ERR_ARG, "border must not be negative");
	if (c->skin > 0.0) return set_error(c, MDGPU_ERR_STATE, "the coupling operations need the per-step binning (skin 0)");
	if (c->n == 0) return set_error(c, MDGPU_ERR_STATE, "no molecules loaded");
	cudaError_t e = cudaSetDevice(c->device);
	if (e == cudaSuccess) {
		k_force_boundary<<<nblk(c->n), kT, 0, c->stream>>>(c->n, c->p, c->g, dim, border, stream_out_dir, stream_damping);
		count_launches(c, 1);
		e = cudaGetLastError();
	}
	if (e != cudaSuccess) return set_cuda_error(c, e, "mdgpu_force_boundary");
	return check_device_status(c);
}

int mdgpu_thermostat_create(mdgpu_thermostat** out, mdgpu_ctx* ctx, const mdgpu_coupling_cells* cells,
                            double target_temperature, double gamma, int32_t interval, const int32_t directed[3]) {
	if (!out || !ctx || !cells || !directed) return MDGPU_ERR_ARG;
	*out = nullptr;
	Context* c = &ctx->c;
	if (cells->dim != 2 && cells->dim != 3) return set_error(c, MDGPU_ERR_ARG, "dim must be 2 or 3");
	if (!(cells->cell_size > 0.0)) return set_error(c, MDGPU_ERR_ARG, "cell_size must be positive");
	int64_t ncells = 1;
	for (int d = 0; d < 3; d++) {
		if (cells->size[d] < 1) return set_error(c, MDGPU_ERR_ARG, "cells per dimension must be >= 1");
		ncells *= cells->size[d];
	}
	if (cells->dim == 2 && cells->size[2] != 1) return set_error(c, MDGPU_ERR_ARG, "two-dimensional grids have size[2] 1");
	if (ncells > (1 << 26)) return set_error(c, MDGPU_ERR_ARG, "too many coupling cells");
	if (interval < 0) return set_error(c, MDGPU_ERR_ARG, "interval must not be negative");
	mdgpu_thermostat* th = new (std::nothrow) mdgpu_thermostat();
	if (!th) return MDGPU_ERR_ARG;
	th->ctx = ctx;
	th->device = c->device;
	for (int d = 0; d < 3; d++) {
		th->cg.lower[d] = cells->lower[d];
		th->cg.upper[d] = cells->upper[d];
		th->cg.size[d] = cells->size[d];
		th->directed[d] = directed[d];
	}
	th->cg.cell = cells->cell_size;
	th->cg.dim = cells->dim;
	th->ncells = (int) ncells;
	th->T = target_temperature;
	th->gamma = gamma;
	th->interval = interval;
	cudaError_t e = cudaSetDevice(c->device);
	// vsum (4), esum (1), shadow (4), vc (3) per cell; everything but vc starts at zero
	const size_t bytes = sizeof(unsigned long long) * 5 * ncells + sizeof(double) * 7 * ncells;
	th->vsum = nullptr;
	if (e == cudaSuccess) e = cudaMalloc(&th->vsum, bytes);
	if (e == cudaSuccess) e = cudaMemsetAsync(th->vsum, 0, bytes, c->stream);
	if (e != cudaSuccess) {
		cudaFree(th->vsum);
		delete th;
		return set_cuda_error(c, e, "mdgpu_thermostat_create");
	}
	th->esum = th->vsum + 4 * ncells;
	th->shadow = reinterpret_cast<double*>(th->esum + ncells);
	th->vc = th->shadow + 4 * ncells;
	*out = th;
	return MDGPU_OK;
}

int mdgpu_thermostat_apply(mdgpu_thermostat* th, int64_t iteration) {
	if (!th) return MDGPU_ERR_ARG;
	Context* c = &th->ctx->c;
	if (c->n == 0) return set_error(c, MDGPU_ERR_STATE, "no molecules loaded");
	cudaError_t e = cudaSetDevice(c->device);
	const int64_t n = c->n;
	if (e == cudaSuccess) {
		k_th_save<<<nblk(n), kT, 0, c->stream>>>(n, c->p, th->cg, th->vsum, th->shadow);
		count_launches(c, 1);
		e = cudaGetLastError();
	}
	if (e == cudaSuccess && th->interval != 0 && iteration % th->interval == 0) {
		k_th_cells<<<nblk(th->ncells), kT, 0, c->stream>>>(th->ncells, th->vsum, th->directed[0], th->directed[1],
		                                                     th->directed[2], th->vc, th->esum, th->shadow, c->status);
		k_th_energy<<<nblk(n), kT, 0, c->stream>>>(n, c->p, th->cg, c->sp, th->vc, th->esum, th->shadow);
		k_th_adjust<<<nblk(n), kT, 0, c->stream>>>(n, c->p, th->cg, th->vsum, th->vc, th->esum, th->shadow, c->status,
		                                           (double) th->interval, th->T, th->gamma);
		count_launches(c, 3);
		e = cudaGetLastError();
		// the next interval's sums start from zero (the energies are cleared by k_th_cells)
		if (e == cudaSuccess) e = cudaMemsetAsync(th->vsum, 0, sizeof(unsigned long long) * 4 * th->ncells, c->stream);
		if (e == cudaSuccess) e = cudaMemsetAsync(th->shadow, 0, sizeof(double) * 4 * th->ncells, c->stream);
	}
	if (e != cudaSuccess) return set_cuda_error(c, e, "mdgpu_thermostat_apply");
	return check_device_status(c);
}

int mdgpu_thermostat_destroy(mdgpu_thermostat* th) {
	if (!th) return MDGPU_OK;
	int prev = -1;
	cudaGetDevice(&prev);
	cudaSetDevice(th->device);
	cudaFree(th->vsum);
	if (prev >= 0) cudaSetDevice(prev);
	delete th;
	return MDGPU_OK;
}

}  // extern "C"
