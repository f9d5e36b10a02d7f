// Single-box pair kernels: one CTA per brick of 2x2x2 linked cells (the per-brick work is in
// brick.cuh, which also documents the staging, filter and compute passes).
//
//   k_pairs_brick  filter + exact evaluation every call (the drop-in traversal)
//   k_build_lists  Verlet-skin mode, build step: each molecule's candidates within rc + skin
//   k_pairs_list   Verlet-skin mode, every step: exact evaluation of the lists at the current
//                  positions
// In the Verlet-skin mode the build is launched every step and returns at once unless a device flag
// (set by the Leapfrog pre-kick when a molecule moved more than skin/2 since the build) is set.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>

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
                  double* __restrict__ partials, int* __restrict__ status, const int* __restrict__ gate,
                  brick::Lists lists) {
	extern __shared__ __align__(16) unsigned char smem[];
	brick::load_params(smem, brick::layout(p.s_cap, kFP64, kListCap), pp, p.ns);
	__syncthreads();
	brick::pairs<kFP64, kSingle, kLjIsRc, kListCap>(p, bx, blockIdx.x, blockIdx.x, smem, rx, ry, rz, cid, cstart, fx,
	                                                fy, fz, partials, status);
}

// Verlet-skin build step (runs only when *gate is this step's id): the lists, no forces.
__global__ void __launch_bounds__(brick::kThreads, 3)
    k_build_lists(brick::Box bx, int nbricks, int s_cap, const double* __restrict__ rx,
                  const double* __restrict__ ry, const double* __restrict__ rz, const int32_t* __restrict__ cstart,
                  const int* __restrict__ gate, int step, brick::Lists lists) {
	if (*gate != step) return;
	if (lists.pst && blockIdx.x == 0 && threadIdx.x == 0) lists.pst->built = step;   // pruned lists: prune now
	extern __shared__ __align__(16) unsigned char smem[];
	// a resident grid walks the bricks: a step without a build costs one launch of that grid only
	for (int b = blockIdx.x; b < nbricks; b += gridDim.x) {
		brick::build_lists(bx, b, s_cap, smem, rx, ry, rz, cstart, lists, b);
		__syncthreads();
	}
}

#ifndef MDGPU_LIST_MINB
#define MDGPU_LIST_MINB 3
#endif
// Resident CTAs per SM of the FP32 list kernel (registers and shared memory are sized for it).
constexpr int kListMinBlocks = MDGPU_LIST_MINB;

// The list evaluation of a step. With pruned lists (lists.pst set) it comes in two variants, launched
// one after the other in every step: kPrune runs in the steps that prune (the lists were built in
// this step, or the summed largest drifts since the last prune reached half_prune), reads the build
// lists and writes the inner lists (po) besides the forces; the plain variant runs in the other
// steps and reads the inner lists. Both decide from values that no CTA of their launch changes (not
// from the rebuild flag, which the fused kick of this step may set for the next one).
template <bool kFP64, bool kSingle, bool kLjIsRc, bool kPrune = false>
__global__ void __launch_bounds__(brick::kThreads, kFP64 ? 2 : kListMinBlocks)
    k_pairs_list(brick::Const p, brick::Box bx, const double* __restrict__ rx, const double* __restrict__ ry,
                 const double* __restrict__ rz, const int32_t* __restrict__ cid,
                 const int32_t* __restrict__ cstart, const PairParams* __restrict__ pp,
                 double* __restrict__ fx, double* __restrict__ fy, double* __restrict__ fz,
                 double* __restrict__ partials, int* __restrict__ status, const int* __restrict__ gate,
                 brick::Lists lists, unsigned* tickets, double* scalars, brick::Kick kick, double* record,
                 brick::PruneOut po, double half_prune) {
	if (lists.pst) {
		const PruneState* st = lists.pst;
		if (kPrune) {
			const double moved = st->acc + sqrt((double) __uint_as_float(st->dmax[lists.step & 1]));
			if (st->built != lists.step && moved < half_prune) return;
			if (blockIdx.x == 0 && threadIdx.x == 0) {
				lists.pst->pruned = lists.step;
				lists.pst->count++;
			}
		} else if (st->pruned == lists.step) {
			return;   // the prune variant evaluated this step
		}
	}
	extern __shared__ __align__(16) unsigned char smem[];
	__shared__ int s_item;
	brick::load_params(smem, brick::layout(p.s_cap, kFP64, 0, false), pp, p.ns);
	if (threadIdx.x == 0) brick::drift_slot() = 0u;   // read after the barriers below
	if (lists.kind == nullptr) {
		// every brick, one CTA each
		__syncthreads();
		brick::list_pairs<kFP64, kSingle, kLjIsRc, true, kPrune>(p, bx, blockIdx.x, blockIdx.x, smem, rx, ry, rz, cid,
		                                                         cstart, fx, fy, fz, partials, status, lists, kick, po);
	} else {
		// the dense bricks of the last build (the sparse ones go to k_pairs_list_sparse): a resident
		// grid takes them from a queue
		const int nwork = (int) *(volatile unsigned*) (lists.counts + 1);
		for (;;) {
			__syncthreads();
			if (threadIdx.x == 0) s_item = (int) atomicAdd(lists.counts + 2, 1u);
			__syncthreads();
			const int item = s_item;
			if (item >= nwork) break;
			const int b = lists.blist[item];
			brick::list_pairs<kFP64, kSingle, kLjIsRc, true, kPrune>(p, bx, b, b, smem, rx, ry, rz, cid, cstart, fx, fy,
			                                                         fz, partials, status, lists, kick, po);
		}
	}
	__syncthreads();
	brick::drift_flush(kick.dmax);
	// U6 sum, virial sum, pair count (and sum m v^2 of the closing kick) of the step over every
	// brick's partials, summed by the last CTA to finish, which also writes the step record
	// {Upot, virial, sum m v^2, pairs} and resets both work queues
	if (last_block_sum(tickets, partials, lists.nbricks, kick.mode ? 4 : 3, scalars) && threadIdx.x == 0) {
		lists.counts[2] = 0u;
		lists.counts[3] = 0u;
		if (lists.pst) {
			// the drift into this step's positions joins the sum, which a prune at this step restarts
			PruneState* st = lists.pst;
			const int par = lists.step & 1;
			st->acc = kPrune ? 0.0 : st->acc + sqrt((double) __uint_as_float(st->dmax[par]));
			st->dmax[par] = 0u;
		}
		if (record) {
			record[0] = scalars[0] * 0.5 / 6.;
			record[1] = scalars[1] * 0.5;
			record[2] = scalars[3];
			record[3] = scalars[2] * 0.5;
		}
	}
}

// Sparse bricks (few molecules, e.g. a vapour), one warp each: every warp of a resident grid takes
// the sparse bricks of the last build from a queue.
template <bool kFP64, bool kSingle, bool kLjIsRc>
__global__ void __launch_bounds__(brick::kThreads, 2)
    k_pairs_list_sparse(brick::Const p, brick::Box bx, const double* __restrict__ rx,
                        const double* __restrict__ ry, const double* __restrict__ rz,
                        const int32_t* __restrict__ cid, const int32_t* __restrict__ cstart,
                        const PairParams* __restrict__ pp, double* __restrict__ fx, double* __restrict__ fy,
                        double* __restrict__ fz, double* __restrict__ partials, int* __restrict__ status,
                        brick::Lists lists, brick::Kick kick) {
	extern __shared__ __align__(16) unsigned char smem[];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	unsigned char* ws = smem + warp * brick::sparse_warp_bytes(kFP64);
	const brick::SmemLayout L = brick::layout(brick::kSparseCap, kFP64, 0, false);
	double* pd = reinterpret_cast<double*>(ws + L.params);
	float* pf = reinterpret_cast<float*>(pd + 3 * brick::KK);
	for (int k = lane; k < p.ns * p.ns; k += 32) {
		pd[k] = pp->eps24[k];
		pd[brick::KK + k] = pp->sig2[k];
		pd[2 * brick::KK + k] = pp->shift6[k];
		pf[k] = (float) pp->eps24[k];
		pf[brick::KK + k] = (float) pp->sig2[k];
		pf[2 * brick::KK + k] = (float) pp->shift6[k];
	}
	if (lane == 0)
		reinterpret_cast<float4*>(ws + L.hi)[brick::kSparseCap] =
		    make_float4(1e15f, 1e15f, 1e15f, __uint_as_float((256u << 18) | (256u << 9) | 256u));
	if (threadIdx.x == 0) brick::drift_slot() = 0u;
	__syncthreads();
	const int nwork = (int) *(volatile unsigned*) lists.counts;
	for (;;) {
		__syncwarp();
		int item = 0;
		if (lane == 0) item = (int) atomicAdd(lists.counts + 3, 1u);
		item = __shfl_sync(brick::kFull, item, 0);
		if (item >= nwork) break;
		const int b = lists.blist[lists.nbricks + item];
		brick::list_pairs_warp<kFP64, kSingle, kLjIsRc>(p, bx, b, ws, rx, ry, rz, cid, cstart, fx, fy, fz, partials,
		                                                status, lists, kick);
	}
	__syncthreads();
	brick::drift_flush(kick.dmax);
}

// Resident grid of a kernel: the CTAs that fit on the device at once (at most `cap`). The
// occupancy query is a host call of several microseconds; its answer per (kernel, shared memory)
// is kept, since small boxes stepped one launch at a time would otherwise pay it every step.
template <typename K>
int resident_grid(const Context* c, K kern, size_t smem, int cap) {
	static std::mutex mu;
	static std::map<std::pair<const void*, size_t>, int> known;
	const auto key = std::make_pair(reinterpret_cast<const void*>(kern), smem);
	int per_sm = 0;
	{
		std::lock_guard<std::mutex> lock(mu);
		auto it = known.find(key);
		if (it != known.end()) per_sm = it->second;
	}
	if (per_sm == 0) {
		if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, brick::kThreads, smem) != cudaSuccess ||
		    per_sm < 1)
			per_sm = 1;
		std::lock_guard<std::mutex> lock(mu);
		known[key] = per_sm;
	}
	return std::max(1, std::min(cap, per_sm * c->num_sms));
}

struct Plan {
	brick::Const p;
	brick::Box bx;
	size_t bytes;
	int nbricks;
};

// kind 0: plain traversal, 2: list evaluation of the skin mode (two CTAs per SM).
Plan plan(Context* c, const Grid& g, double filter_radius, int kind) {
	const bool fp64 = c->precision == MDGPU_FP64;
	Plan P;
	brick::init_box(P.bx, g, filter_radius, 0, kind == 0 ? 0.0 : 0.5 * c->skin);
	const int max_optin = device_max_optin(c->device);
	size_t budget = 110 * 1024;
	if (kind == 2 && !fp64) budget = std::min(budget, (size_t) (224 / kListMinBlocks - 2) * 1024);
	if (kind == 2 && pruning(c)) budget -= brick::kPruneRingBytes;   // the prune variant's ring
	if (budget > (size_t) max_optin) budget = (size_t) max_optin;
	const int lcap = kind == 2 ? 0 : kListCap;
	const bool half = kind != 2;
	const int s_cap = brick::capacity_for(budget, fp64, lcap, half);
	P.p = brick::make_const(c->sp.n, s_cap, c->rc, c->rc_lj);
	P.bytes = brick::layout(s_cap, fp64, lcap, half).total;
	P.nbricks = P.bx.nb[0] * P.bx.nb[1] * P.bx.nb[2];
	return P;
}

template <typename K, typename... Extra>
cudaError_t go(Context* c, const Plan& P, K kern, const int* gate, const brick::Lists& lists, Extra... extra) {
	cudaError_t r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) P.bytes);
	// the list kernel runs as a resident grid over a queue of the dense bricks when the sparse ones
	// are evaluated apart (lists.kind set); otherwise one CTA per brick
	const int grid = lists.kind && sizeof...(Extra) > 0 ? resident_grid(c, kern, P.bytes, P.nbricks) : P.nbricks;
	if (r == cudaSuccess)
		kern<<<grid, brick::kThreads, P.bytes, c->stream>>>(P.p, P.bx, c->p.rx, c->p.ry, c->p.rz, c->p.cid,
		                                                         c->cell_start, c->d_pp, c->p.fx, c->p.fy, c->p.fz,
		                                                         c->partials, c->status, gate, lists, extra...);
	return r;
}

// kind 0: plain traversal, 2: list evaluation of the skin mode (kPr: its prune variant)
template <int kKind, bool kPr = false>
cudaError_t dispatch(Context* c, const Plan& P, const int* gate, const brick::Lists& lists,
                     const brick::Kick& kick = brick::Kick{}, double* record = nullptr,
                     const brick::PruneOut& po = brick::PruneOut{}, double half_prune = 0.0) {
	const bool fp64 = c->precision == MDGPU_FP64;
	const bool single = c->sp.n == 1, ljrc = c->rc_lj == c->rc;
	if (kKind == 2) {
		unsigned* t = c->tickets;
		double* out = c->scalars;
		if (fp64)
			return single ? go(c, P, k_pairs_list<true, true, false, kPr>, gate, lists, t, out, kick, record, po, half_prune)
			              : go(c, P, k_pairs_list<true, false, false, kPr>, gate, lists, t, out, kick, record, po,
			                   half_prune);
		if (ljrc)
			return single ? go(c, P, k_pairs_list<false, true, true, kPr>, gate, lists, t, out, kick, record, po, half_prune)
			              : go(c, P, k_pairs_list<false, false, true, kPr>, gate, lists, t, out, kick, record, po,
			                   half_prune);
		return single ? go(c, P, k_pairs_list<false, true, false, kPr>, gate, lists, t, out, kick, record, po, half_prune)
		              : go(c, P, k_pairs_list<false, false, false, kPr>, gate, lists, t, out, kick, record, po,
		                   half_prune);
	}
	if (fp64) return single ? go(c, P, k_pairs_brick<true, true, false>, gate, lists)
	                        : go(c, P, k_pairs_brick<true, false, false>, gate, lists);
	if (ljrc) return single ? go(c, P, k_pairs_brick<false, true, true>, gate, lists)
	                        : go(c, P, k_pairs_brick<false, false, true>, gate, lists);
	return single ? go(c, P, k_pairs_brick<false, true, false>, gate, lists)
	              : go(c, P, k_pairs_brick<false, false, false>, gate, lists);
}

brick::Lists lists_of(Context* c) {
	brick::Lists l{};
	l.nbr = c->nbr;
	l.count = c->nbr_count;
	l.rx_ref = c->r_ref;
	l.ry_ref = c->r_ref + c->n;
	l.rz_ref = c->r_ref + 2 * c->n;
	l.n = c->n;
	l.cap = c->list_cap;
	l.builds = c->builds;
	l.kind = c->brick_kind;
	l.counts = c->brick_counts;
	l.blist = c->brick_list;
	l.nbricks = (int) skin_partials_needed(c);
	return l;
}

}  // namespace

cudaError_t launch_pairs_brick(Context* c) {
	const Plan P = plan(c, c->g, c->rc, 0);
	prof_begin(c, 1);
	cudaError_t e = dispatch<0>(c, P, nullptr, brick::Lists{});
	if (e == cudaSuccess) e = cudaGetLastError();
	prof_end(c, 1, 1);
	if (e != cudaSuccess) return e;
	return launch_reduce(c, P.nbricks, c->scalars, 3);
}

cudaError_t launch_pairs_skin(Context* c, int kick_mode, double dt, double* record) {
	brick::Lists l = lists_of(c);
	brick::Kick kick{};
	kick.mode = kick_mode;
	if (kick_mode) {
		kick.id = c->step_id + 1;   // the step whose rebuild a long drift asks for
		kick.dt = dt;
		kick.half2 = 0.25 * c->skin * c->skin;
		for (int k = 0; k < c->sp.n; k++) {
			kick.post[k] = (0.5 * dt) / c->sp.mass[k];
			kick.pre[k] = (.5 * dt) / c->sp.mass[k];
			kick.mass[k] = c->sp.mass[k];
		}
		kick.vx = c->p.vx;
		kick.vy = c->p.vy;
		kick.vz = c->p.vz;
		kick.ox = c->q.rx;
		kick.oy = c->q.ry;
		kick.oz = c->q.rz;
		kick.flag = c->rebuild;
		if (pruning(c) && kick_mode == 1) kick.dmax = &c->prune_st->dmax[(c->step_id + 1) & 1];
	}
	const Plan P = plan(c, c->gs, c->rc, 2);
	l.sentinel = P.p.s_cap;   // the evaluation kernel's sentinel slot terminates every list
	int launches = 2;
	// pruned lists: the prune variant of the evaluation reads the build lists (and writes the inner
	// ones) in the steps that prune, the plain variant reads the inner lists in the others; the
	// sparse bricks always evaluate their build lists; the build records its step in the prune state
	brick::Lists inner = l;
	brick::PruneOut po{};
	double half_prune = 0.0;
	const bool prune = pruning(c);
	if (prune) {
		l.pst = c->prune_st;
		l.step = c->step_id;
		inner = l;
		inner.nbr = c->nbr_in;
		inner.count = c->nbr_in_count;
		po.nbr = c->nbr_in;
		po.count = c->nbr_in_count;
		// the FP64 form tests the staged hi parts only: the lo parts (at most 256 steps each way
		// per coordinate, plus half a step of quantisation) move the distance by at most
		// sqrt(3) * 513 steps; the float arithmetic by a few 1e-7 of it
		const double lo = 520.0 * std::max(P.bx.lo_step[0], std::max(P.bx.lo_step[1], P.bx.lo_step[2]));
		const double rp = c->rc + c->prune + 1.7320508075688772 * lo;
		const double rp2 = rp * rp * (1.0 + 2e-6);
		po.rp2f = (float) rp2;
		if ((double) po.rp2f < rp2) po.rp2f = std::nextafter(po.rp2f, 2.0f * po.rp2f);
		// prune when the drifts reach half the inner skin, less a margin that keeps every pair left
		// out farther than rc (1 + 1e-5) from the other molecule until then
		half_prune = 0.5 * c->prune - 1e-5 * (c->rc + c->prune);
		launches++;
	}
	prof_begin(c, 1);
	// build (gated): half-precision staging only, three CTAs per SM
	brick::Box bb{};
	brick::init_box(bb, c->gs, c->rc + c->skin, 0, 0.5 * c->skin);
	int s_cap = 256;
	while (brick::build_bytes(s_cap + 64) <= 72 * 1024) s_cap += 64;
	const size_t bbytes = brick::build_bytes(s_cap);
	const int nbricks = bb.nb[0] * bb.nb[1] * bb.nb[2];
	cudaError_t e = cudaFuncSetAttribute(k_build_lists, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bbytes);
	const int grid = std::min(nbricks, 3 * c->num_sms);   // three CTAs per SM (launch bounds, 72 KB each)
	if (e == cudaSuccess)
		k_build_lists<<<grid, brick::kThreads, bbytes, c->stream>>>(bb, nbricks, s_cap, c->p.rx, c->p.ry, c->p.rz,
		                                                           c->cell_start, c->rebuild, c->step_id, l);
	// evaluation, every step: sparse bricks one warp each, then the others (whose last CTA sums the
	// partials of all bricks). When the last build of an earlier run found no sparse brick the
	// dense kernel takes every brick (kind not consulted) and the sparse kernel is not launched.
	const bool sparse = !c->h_sparse || *(volatile int*) c->h_sparse != 0;
	brick::Lists ld = l, ldi = inner;
	if (!sparse) ld.kind = ldi.kind = nullptr;
	if (e == cudaSuccess && sparse) {
		const bool fp64 = c->precision == MDGPU_FP64;
		const bool single = c->sp.n == 1, ljrc = c->rc_lj == c->rc;
		auto ks = fp64 ? (single ? k_pairs_list_sparse<true, true, false> : k_pairs_list_sparse<true, false, false>)
		               : (single ? (ljrc ? k_pairs_list_sparse<false, true, true> : k_pairs_list_sparse<false, true, false>)
		                         : (ljrc ? k_pairs_list_sparse<false, false, true>
		                                 : k_pairs_list_sparse<false, false, false>));
		const size_t sbytes = brick::kWarps * brick::sparse_warp_bytes(fp64);
		const brick::Const ps = brick::make_const(c->sp.n, brick::kSparseCap, c->rc, c->rc_lj);
		e = cudaFuncSetAttribute(ks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sbytes);
		const int sgrid = resident_grid(c, ks, sbytes, (P.nbricks + brick::kWarps - 1) / brick::kWarps);
		if (e == cudaSuccess)
			ks<<<sgrid, brick::kThreads, sbytes, c->stream>>>(ps, P.bx, c->p.rx, c->p.ry, c->p.rz, c->p.cid,
			                                                   c->cell_start, c->d_pp, c->p.fx, c->p.fy, c->p.fz,
			                                                   c->partials, c->status, l, kick);
	}
	if (e == cudaSuccess && prune) {
		Plan Pp = P;
		Pp.bytes += brick::kPruneRingBytes;
		e = dispatch<2, true>(c, Pp, nullptr, ld, kick, record, po, half_prune);
	}
	if (e == cudaSuccess) e = dispatch<2>(c, P, nullptr, prune ? ldi : ld, kick, record);
	if (e == cudaSuccess) e = cudaGetLastError();
	prof_end(c, 1, sparse ? launches + 1 : launches);
	return e;
}

int64_t skin_partials_needed(const Context* c) {
	return (int64_t) ((c->gs.nc[0] + 1) / 2) * ((c->gs.nc[1] + 1) / 2) * ((c->gs.nc[2] + 1) / 2);
}

}  // namespace mdgpu
