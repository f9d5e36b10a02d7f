// Reverse-mode gradient through an NVE Leapfrog trajectory, entirely on the device, with the
// checkpoints kept as device snapshots: mdgpu_traj_forward / mdgpu_traj_backward. No counterpart
// in the reference (it has no gradients); the forward step is the reference's
// (Simulation::simulateStep with Leapfrog, Simulation.cpp:1218-1229, Leapfrog.cpp:37-99, paths
// relative to madpac/mardyn/), NVE, vcorr = 1:
//
//   v_h = v_k + c F_k,   r_{k+1} = r_k + dt v_h,   F_{k+1} = F(r_{k+1}),   v_{k+1} = v_h + c F_{k+1}
//
// with c = dt / (2 m). Backwards, for cotangents (rbar, vbar, Fbar) of the state after step k+1:
//
//   Fbar += c vbar                         (F_{k+1} reaches L through v_{k+1})
//   rbar += J(r_{k+1})^T Fbar (+ the energy cotangent at the final step)   (k_adjoint)
//   vbar  = vbar + dt rbar                 (through r_{k+1} = r_k + dt v_h, and v_h = v_k + ...)
//   Fbar  = c vbar                         (F_k reaches L through v_h)
//
// and at the start rbar += J(r_0)^T Fbar. The forward pass keeps (r, v) every `every` steps
// (caller order, device memory); the backward pass recomputes each segment from its snapshot,
// keeping the segment's positions, and walks it backwards. Nothing goes through host memory but
// the cotangents in and the gradients out.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "md_internal.h"

namespace mdgpu {

cudaError_t launch_adjoint(Context* c, const double* gfx, const double* gfy, const double* gfz, double gU, double* ox,
                           double* oy, double* oz, double* pgrad, double* pout, bool accumulate);
int check_device_status(Context* c);

namespace {

constexpr int kT = 256;
constexpr int KK = kMaxSpecies * kMaxSpecies;

inline unsigned nblk(int64_t n) { return (unsigned) ((n + kT - 1) / kT); }

// sorted arrays -> caller order (SoA planes of n doubles each)
__global__ void k_snap(int64_t n, const int32_t* __restrict__ uidx, const double* __restrict__ x,
                       const double* __restrict__ y, const double* __restrict__ z, double* __restrict__ dst) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const int64_t u = uidx[s];
	dst[u] = x[s];
	dst[n + u] = y[s];
	dst[2 * n + u] = z[s];
}

// caller order -> the sorted arrays of the current order
__global__ void k_restore(int64_t n, const int32_t* __restrict__ uidx, const double* __restrict__ src,
                          double* __restrict__ x, double* __restrict__ y, double* __restrict__ z) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const int64_t u = uidx[s];
	x[s] = src[u];
	y[s] = src[n + u];
	z[s] = src[2 * n + u];
}

// c = dt/(2m) per molecule in caller order
__global__ void k_cmol(int64_t n, const int32_t* __restrict__ uidx, const int32_t* __restrict__ cid, Species sp,
                       double dt, double* __restrict__ cm) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	cm[uidx[s]] = (0.5 * dt) / sp.mass[cid[s]];
}

// Fbar += c vbar (when `with_v`), and Fbar in the sorted order for the adjoint kernel
__global__ void k_vjp_in(int64_t n, const int32_t* __restrict__ uidx, const double* __restrict__ cm,
                         const double* __restrict__ vbar, double* __restrict__ Fbar, bool with_v,
                         double* __restrict__ gx, double* __restrict__ gy, double* __restrict__ gz) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const int64_t u = uidx[s];
	double f[3];
	for (int d = 0; d < 3; d++) {
		f[d] = Fbar[d * n + u];
		if (with_v) f[d] += cm[u] * vbar[d * n + u];
		Fbar[d * n + u] = f[d];
	}
	gx[s] = f[0];
	gy[s] = f[1];
	gz[s] = f[2];
}

// rbar += J^T Fbar (sorted -> caller order); with `step`: vbar = vbar + dt rbar, Fbar = c vbar
__global__ void k_vjp_out(int64_t n, const int32_t* __restrict__ uidx, const double* __restrict__ cm, double dt,
                          const double* __restrict__ ox, const double* __restrict__ oy, const double* __restrict__ oz,
                          double* __restrict__ rbar, double* __restrict__ vbar, double* __restrict__ Fbar, bool step) {
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const int64_t u = uidx[s];
	const double o[3] = {ox[s], oy[s], oz[s]};
	for (int d = 0; d < 3; d++) {
		const double rb = rbar[d * n + u] + o[d];
		rbar[d * n + u] = rb;
		if (step) {
			const double vb = vbar[d * n + u] + dt * rb;
			vbar[d * n + u] = vb;
			Fbar[d * n + u] = cm[u] * vb;
		}
	}
}

// caller-order planes (SoA) <-> (n, 3) rows
__global__ void k_planes_to_rows(int64_t n, const double* __restrict__ src, double* __restrict__ dst) {
	const int64_t u = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (u >= n) return;
	dst[3 * u] = src[u];
	dst[3 * u + 1] = src[n + u];
	dst[3 * u + 2] = src[2 * n + u];
}

__global__ void k_rows_to_planes(int64_t n, const double* __restrict__ src, double* __restrict__ dst) {
	const int64_t u = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (u >= n) return;
	dst[u] = src[3 * u];
	dst[n + u] = src[3 * u + 1];
	dst[2 * n + u] = src[3 * u + 2];
}

}  // namespace

// Device buffers of a trajectory (one per context).
struct Traj {
	int64_t n = 0;
	int nsteps = 0, every = 0;
	double dt = 0.0;
	std::vector<int> starts;   // checkpointed steps
	double* snaps = nullptr;   // starts.size() x (r, v) planes (6 n)
	double* seg = nullptr;     // (every + 1) x r planes (3 n)
	double *rbar = nullptr, *vbar = nullptr, *Fbar = nullptr, *cm = nullptr;
	double *gs = nullptr, *os = nullptr, *pgrad = nullptr, *par = nullptr, *rows = nullptr;
	int64_t cap_snaps = 0, cap_seg = 0, cap_n = 0;
	int64_t recomputed = 0;
	bool valid = false;
	// with the context's profiling on: events around each adjoint launch of the last backward pass
	std::vector<cudaEvent_t> ev;
	double adj_ms = 0.0;
	int64_t adj_launches = 0;
	~Traj() {
		cudaFree(snaps);
		cudaFree(seg);
		cudaFree(rbar);
		cudaFree(gs);
		for (cudaEvent_t e : ev) cudaEventDestroy(e);
	}
};

void free_traj(Context* c) {
	delete c->traj;
	c->traj = nullptr;
}

namespace {

// The binning of every step: the cooperative rebuild in its always-build form, one launch (the
// same (cell, id) order as launch_bin's six kernels).
cudaError_t traj_bin(Context* c) { return launch_rebuild(c, c->g, nullptr, nullptr, 0, true); }

// One reference step (NVE) on the context: pre-kick and drift, binning, forces, closing kick.
cudaError_t traj_step(Context* c, double dt) {
	cudaError_t e = launch_leapfrog_pre(c, dt, 1.0);
	if (e == cudaSuccess) e = traj_bin(c);
	if (e == cudaSuccess) e = launch_pairs(c);
	if (e == cudaSuccess) e = launch_leapfrog_post(c, 0.5 * dt);
	return e;
}

cudaError_t traj_snap(Context* c, double* dst, bool with_v) {
	const int64_t n = c->n;
	k_snap<<<nblk(n), kT, 0, c->stream>>>(n, c->p.uidx, c->p.rx, c->p.ry, c->p.rz, dst);
	if (with_v) k_snap<<<nblk(n), kT, 0, c->stream>>>(n, c->p.uidx, c->p.vx, c->p.vy, c->p.vz, dst + 3 * n);
	count_launches(c, with_v ? 2 : 1);
	return cudaGetLastError();
}

cudaError_t traj_restore(Context* c, const double* src, bool with_v) {
	const int64_t n = c->n;
	k_restore<<<nblk(n), kT, 0, c->stream>>>(n, c->p.uidx, src, c->p.rx, c->p.ry, c->p.rz);
	if (with_v) k_restore<<<nblk(n), kT, 0, c->stream>>>(n, c->p.uidx, src + 3 * n, c->p.vx, c->p.vy, c->p.vz);
	count_launches(c, with_v ? 2 : 1);
	return cudaGetLastError();
}

// J^T Fbar at the positions now in the context (binned), accumulated into rbar (and, with `step`,
// the Leapfrog part of the backward step); parameter terms added to t->par.
cudaError_t traj_vjp(Context* c, Traj* t, double gU, bool with_v, bool step) {
	const int64_t n = c->n;
	double *gx = t->gs, *gy = gx + n, *gz = gy + n, *ox = t->os, *oy = ox + n, *oz = oy + n;
	k_vjp_in<<<nblk(n), kT, 0, c->stream>>>(n, c->p.uidx, t->cm, t->vbar, t->Fbar, with_v, gx, gy, gz);
	count_launches(c, 1);
	cudaEvent_t a = nullptr, b = nullptr;
	if (c->profiling) {
		cudaEventCreate(&a);
		cudaEventCreate(&b);
		t->ev.push_back(a);
		t->ev.push_back(b);
		cudaEventRecord(a, c->stream);
	}
	cudaError_t e = launch_adjoint(c, gx, gy, gz, gU, ox, oy, oz, t->pgrad, t->par, true);
	if (c->profiling) cudaEventRecord(b, c->stream);
	if (e != cudaSuccess) return e;
	k_vjp_out<<<nblk(n), kT, 0, c->stream>>>(n, c->p.uidx, t->cm, t->dt, ox, oy, oz, t->rbar, t->vbar, t->Fbar, step);
	count_launches(c, 1);
	return cudaGetLastError();
}

}  // namespace
}  // namespace mdgpu

using namespace mdgpu;

extern "C" {

int mdgpu_traj_forward(mdgpu_ctx* ctx, int32_t nsteps, int32_t checkpoint_every, double dt, double* upot_final) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (c->n == 0) return set_error(c, MDGPU_ERR_STATE, "no molecules loaded");
	if (c->skin > 0.0) return set_error(c, MDGPU_ERR_STATE, "the trajectory adjoint needs the per-step binning (skin 0)");
	if (nsteps < 1 || checkpoint_every < 1) return set_error(c, MDGPU_ERR_ARG, "nsteps and checkpoint_every must be >= 1");
	if (!(dt > 0.0)) return set_error(c, MDGPU_ERR_ARG, "dt must be positive");
	cudaError_t e = cudaSetDevice(c->device);
	if (e != cudaSuccess) return set_cuda_error(c, e, "cudaSetDevice");
	{
		const int st = rebuild_prepare(c);   // the buffers of the per-step binning (traj_bin)
		if (st) return st;
	}
	if (!c->traj) c->traj = new Traj();
	Traj* t = c->traj;
	const int64_t n = c->n;
	t->n = n;
	t->nsteps = nsteps;
	t->every = std::min(checkpoint_every, nsteps);
	t->dt = dt;
	t->starts.clear();
	for (int k = 0; k < nsteps; k += t->every) t->starts.push_back(k);
	const int64_t nb = adjoint_blocks(n);
	const int64_t need_snaps = (int64_t) t->starts.size() * 6 * n;
	const int64_t need_seg = (int64_t) (t->every + 1) * 3 * n;
	if (need_snaps > t->cap_snaps) {
		cudaFree(t->snaps);
		t->snaps = nullptr;
		e = cudaMalloc(&t->snaps, sizeof(double) * need_snaps);
		if (e != cudaSuccess) return set_cuda_error(c, e, "cudaMalloc (trajectory snapshots)");
		t->cap_snaps = need_snaps;
	}
	if (need_seg > t->cap_seg) {
		cudaFree(t->seg);
		t->seg = nullptr;
		e = cudaMalloc(&t->seg, sizeof(double) * need_seg);
		if (e != cudaSuccess) return set_cuda_error(c, e, "cudaMalloc (trajectory segment)");
		t->cap_seg = need_seg;
	}
	if (n > t->cap_n) {
		cudaFree(t->rbar);
		cudaFree(t->gs);
		t->rbar = t->gs = nullptr;
		// rbar, vbar, Fbar (3n each), cm (n), rows (3n); gs, os (3n each), pgrad, par
		e = cudaMalloc(&t->rbar, sizeof(double) * 13 * n);
		if (e == cudaSuccess) e = cudaMalloc(&t->gs, sizeof(double) * (6 * n + nb * 2 * KK + 2 * KK));
		if (e != cudaSuccess) return set_cuda_error(c, e, "cudaMalloc (trajectory cotangents)");
		t->cap_n = n;
	}
	t->vbar = t->rbar + 3 * n;
	t->Fbar = t->vbar + 3 * n;
	t->cm = t->Fbar + 3 * n;
	t->rows = t->cm + n;
	t->os = t->gs + 3 * n;
	t->pgrad = t->os + 3 * n;
	t->par = t->pgrad + nb * 2 * KK;
	// forces of the start, then the steps; every `every` steps a snapshot (r, v)
	e = traj_bin(c);
	if (e == cudaSuccess) e = launch_pairs(c);
	if (e == cudaSuccess) e = traj_snap(c, t->snaps, true);
	size_t si = 1;
	for (int k = 1; k <= nsteps && e == cudaSuccess; k++) {
		e = traj_step(c, dt);
		if (e == cudaSuccess && si < t->starts.size() && t->starts[si] == k) e = traj_snap(c, t->snaps + 6 * n * si++, true);
	}
	if (e != cudaSuccess) return set_cuda_error(c, e, "trajectory forward");
	double sc[3];
	e = cudaMemcpyAsync(sc, c->scalars, sizeof(sc), cudaMemcpyDeviceToHost, c->stream);
	if (e != cudaSuccess) return set_cuda_error(c, e, "cudaMemcpyAsync");
	const int st = check_device_status(c);
	if (st) return st;
	c->cells_valid = true;
	t->valid = true;
	if (upot_final) *upot_final = sc[0] * 0.5 / 6.;   // ParticlePairs2PotForceAdapter::finish, both sides
	return MDGPU_OK;
}

int mdgpu_traj_backward(mdgpu_ctx* ctx, const double* gF, double gU, double* dL_dr0, double* dL_dv0, double* dL_deps,
                        double* dL_dsigma, int64_t* recomputed_steps) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	Traj* t = c->traj;
	if (!t || !t->valid || t->n != c->n) return set_error(c, MDGPU_ERR_STATE, "run mdgpu_traj_forward first");
	if (!gF || !dL_dr0) return set_error(c, MDGPU_ERR_ARG, "gF and dL_dr0 are required");
	cudaError_t e = cudaSetDevice(c->device);
	if (e != cudaSuccess) return set_cuda_error(c, e, "cudaSetDevice");
	const int64_t n = c->n;
	const double dt = t->dt;
	// cotangents of the final state: Fbar = gF, rbar = vbar = 0; parameter sums 0
	e = cudaMemcpyAsync(t->rows, gF, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream);
	if (e == cudaSuccess) {
		k_rows_to_planes<<<nblk(n), kT, 0, c->stream>>>(n, t->rows, t->Fbar);
		count_launches(c, 1);
		e = cudaMemsetAsync(t->rbar, 0, sizeof(double) * 6 * n, c->stream);
	}
	if (e == cudaSuccess) e = cudaMemsetAsync(t->par, 0, sizeof(double) * 2 * KK, c->stream);
	if (e == cudaSuccess) {
		k_cmol<<<nblk(n), kT, 0, c->stream>>>(n, c->p.uidx, c->p.cid, c->sp, dt, t->cm);
		count_launches(c, 1);
	}
	double gUk = gU;
	t->recomputed = 0;
	for (cudaEvent_t ev : t->ev) cudaEventDestroy(ev);
	t->ev.clear();
	for (int si = (int) t->starts.size() - 1; si >= 0 && e == cudaSuccess; si--) {
		const int k0 = t->starts[si];
		const int k1 = si + 1 < (int) t->starts.size() ? t->starts[si + 1] : t->nsteps;
		// the segment from its snapshot: forces of r_k0, then steps k0+1 .. k1, positions kept
		e = traj_restore(c, t->snaps + 6 * n * si, true);
		if (e == cudaSuccess) e = traj_bin(c);
		if (e == cudaSuccess) e = launch_pairs(c);
		for (int k = k0 + 1; k <= k1 && e == cudaSuccess; k++) {
			e = traj_step(c, dt);
			if (e == cudaSuccess) e = traj_snap(c, t->seg + 3 * n * (k - k0), false);
			t->recomputed++;
		}
		// backwards through the segment: F_k = F(r_k) for k = k1 .. k0 + 1
		for (int k = k1; k > k0 && e == cudaSuccess; k--) {
			e = traj_restore(c, t->seg + 3 * n * (k - k0), false);
			if (e == cudaSuccess) e = traj_bin(c);
			if (e == cudaSuccess) e = traj_vjp(c, t, gUk, true, true);
			gUk = 0.0;
		}
	}
	// the start: rbar += J(r_0)^T Fbar
	if (e == cudaSuccess) e = traj_restore(c, t->snaps, true);
	if (e == cudaSuccess) e = traj_bin(c);
	if (e == cudaSuccess) e = traj_vjp(c, t, gUk, false, false);
	double par[2 * KK];
	if (e == cudaSuccess) {
		k_planes_to_rows<<<nblk(n), kT, 0, c->stream>>>(n, t->rbar, t->rows);
		count_launches(c, 1);
		e = cudaMemcpyAsync(dL_dr0, t->rows, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->stream);
	}
	if (e == cudaSuccess && dL_dv0) {
		k_planes_to_rows<<<nblk(n), kT, 0, c->stream>>>(n, t->vbar, t->rows + 0);
		count_launches(c, 1);
		e = cudaMemcpyAsync(dL_dv0, t->rows, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->stream);
	}
	if (e == cudaSuccess) e = cudaMemcpyAsync(par, t->par, sizeof(par), cudaMemcpyDeviceToHost, c->stream);
	if (e != cudaSuccess) return set_cuda_error(c, e, "trajectory backward");
	const int st = check_device_status(c);
	if (st) return st;
	c->cells_valid = true;
	if (recomputed_steps) *recomputed_steps = t->recomputed;
	t->adj_ms = 0.0;
	t->adj_launches = (int64_t) t->ev.size() / 2;
	for (size_t k = 0; k + 1 < t->ev.size(); k += 2) {
		float ms = 0.f;
		if (cudaEventElapsedTime(&ms, t->ev[k], t->ev[k + 1]) == cudaSuccess) t->adj_ms += ms;
	}
	// one parameter per unordered component pair, as mdgpu_adjoint reports them
	const int ns = c->sp.n;
	for (int a = 0; a < ns; a++)
		for (int b = 0; b < ns; b++) {
			const int ab = a * ns + b, ba = b * ns + a;
			const double ge = a == b ? par[ab] : par[ab] + par[ba];
			const double gs = a == b ? par[KK + ab] : par[KK + ab] + par[KK + ba];
			if (dL_deps) dL_deps[ab] = 24.0 * ge;
			if (dL_dsigma) dL_dsigma[ab] = 2.0 * std::sqrt(c->sp.sig2[ab]) * gs;
		}
	return MDGPU_OK;
}

int mdgpu_traj_adjoint_time(mdgpu_ctx* ctx, double* ms, int64_t* launches) {
	if (!ctx) return MDGPU_ERR_ARG;
	Context* c = &ctx->c;
	if (!c->traj) return set_error(c, MDGPU_ERR_STATE, "no trajectory adjoint has run");
	if (ms) *ms = c->traj->adj_ms;
	if (launches) *launches = c->traj->adj_launches;
	return MDGPU_OK;
}

}  // extern "C"
