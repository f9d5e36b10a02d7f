// Internal state of an mdgpu context and the launch helpers shared by the .cu files.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "mdgpu.h"

namespace mdgpu {

constexpr int kMaxSpecies = 8;
constexpr int kMaxDevices = 64;   // device ordinals whose attributes the library caches
constexpr int kReduceBlock = 256;   // block size of every kernel that writes reduction partials

// Device status bits (OR-ed by kernels, mapped to MDGPU_ERR_* by the host).
enum : int {
	kStatusOutsideHalo = 1,
	kStatusSamePosition = 2,
	kStatusNonFinite = 4,
	kStatusTimeout = 8,
	kStatusCapacity = 16,
	kStatusRange = 32,   // a 64-bit fixed-point sum left its range
};

// Comp2Param stream entries per ordered component pair, as doubles and floats.
struct Species {
	int n;
	double eps24[kMaxSpecies * kMaxSpecies];
	double sig2[kMaxSpecies * kMaxSpecies];
	double shift6[kMaxSpecies * kMaxSpecies];
	double mass[kMaxSpecies];
};

// What the pair kernels read: cutoffs and the Comp2Param table (uploaded once per context).
struct PairParams {
	int ns;
	double rc2, rclj2;
	double eps24[kMaxSpecies * kMaxSpecies];
	double sig2[kMaxSpecies * kMaxSpecies];
	double shift6[kMaxSpecies * kMaxSpecies];
};

// Device state of the pruned Verlet-skin lists (mdgpu_set_list_prune). A molecule's inner list
// holds the entries of its build list that were closer than rc + prune at the positions of the
// last prune. Between prunes, acc bounds how far any molecule has moved since then. It is the sum,
// over the drifts, of the largest distance any molecule moved in that drift. A pair left out is
// therefore still beyond rc while 2 acc < prune.
struct PruneState {
	unsigned dmax[2];           // float bits of the largest squared drift of the last step of each parity
	int built;                  // id of the step whose lists were last built (set by the build)
	int pruned;                 // id of the step whose inner lists were last made
	double acc;                 // summed largest drifts since the positions of the last prune
	unsigned long long count;   // prunes so far
};

// LinkedCells geometry. The device keeps only the box's own cells (nc per dimension, no halo
// layer); the reference's halo-inclusive numbering is recovered as inner index + 1 per dimension.
struct Grid {
	int nc[3];
	double L[3];
	double cell_length[3];
	double halo_min[3];
	int64_t ncells;
};

// Particle arrays in cell-sorted order (structure of arrays).
struct Particles {
	double *rx, *ry, *rz;
	double *vx, *vy, *vz;
	double *fx, *fy, *fz;
	uint64_t* id;
	int32_t* cid;
	int32_t* uidx;   // index in the caller's order
};

struct Context {
	int device = 0;
	int num_sms = 148;   // streaming multiprocessors of the device (set at creation)
	cudaStream_t stream = nullptr;
	int precision = MDGPU_FP64;
	int pair_kernel = 0;            // 0 = shared-memory brick kernel, 1 = simple gather kernel
	double rc = 0, rc_lj = 0;
	Grid g{};
	Species sp{};
	double eps[kMaxSpecies], sigma[kMaxSpecies];
	int do_shift[kMaxSpecies];
	double mix[kMaxSpecies * kMaxSpecies];   // xi, eta of each species pair i < j, row by row
	int64_t n = 0;
	int64_t cap = 0;
	bool cells_valid = false;
	std::string err;

	Particles p{};      // current (sorted) arrays
	Particles q{};      // permutation target
	int32_t* cell = nullptr;        // inner cell of each particle (sorted order after update)
	int32_t* rank = nullptr;        // arrival rank within the cell (unordered)
	int32_t* perm = nullptr;        // sorted slot -> previous slot, before the per-cell id sort
	int32_t* cell_count = nullptr;  // ncells
	int32_t* cell_start = nullptr;  // ncells + 1
	int32_t* scan_tmp = nullptr;    // block sums of the scan
	int64_t scan_blocks = 0;
	double* partials = nullptr;     // per-block reduction partials (4 doubles per block)
	int64_t partial_cap = 0;        // in blocks (4 doubles each)
	double* scalars = nullptr;      // device results of the last reductions
	double* steps_out = nullptr;    // per-step results of mdgpu_run / mdgpu_run_async
	int64_t steps_cap = 0;
	int64_t steps_written = 0;      // records appended since the last mdgpu_read_steps
	int* status = nullptr;          // device status word
	unsigned* tickets = nullptr;    // last-block counters of the in-kernel reductions (self-resetting)
	PairParams* d_pp = nullptr;     // device copy of the pair parameters
	// Verlet-skin mode of mdgpu_step / mdgpu_run (skin > 0): per-molecule candidate lists of radius
	// rc + skin on a frozen cell structure, rebuilt (with the binning) by device-side gating when a
	// molecule has moved more than skin/2 since the last build
	double skin = 0.0;
	Grid gs{};                      // cells of edge >= cutoff + skin on which the lists are built
	int max_occ = 0;                // largest cell occupancy of the loaded positions (sizes the lists)
	double rho_typ = 0.0;           // molecule-weighted mean cell density of the loaded positions
	int list_cap = 0;               // list entries per molecule
	int64_t list_n = 0;             // molecules the list buffers hold
	unsigned short* nbr = nullptr;  // list_cap x n staged-slot indices
	unsigned short* nbr_count = nullptr;
	double* r_ref = nullptr;        // 3 x n positions at the last build
	// pruned lists (0 < prune < skin): the entries within rc + prune, which the evaluation reads
	double prune = 0.0;
	unsigned short* nbr_in = nullptr;       // list_cap x n, the layout of nbr
	unsigned short* nbr_in_count = nullptr;
	PruneState* prune_st = nullptr;         // device
	int* rebuild = nullptr;         // device: the step id for which a build was asked
	unsigned char* brick_kind = nullptr;   // per skin-grid brick: 1 = sparse
	int step_id = 0;                // id of the step being enqueued (skin mode)
	unsigned* bar = nullptr;        // grid-barrier words of the cooperative rebuild
	// the cooperative rebuild's cell counts (g.ncells, kept zero between launches) and its per-CTA
	// look-back words (rb_look_cap, kept zero between launches)
	int32_t* rb_count = nullptr;
	unsigned long long* rb_look = nullptr;
	int rb_look_cap = 0;
	// per arrival slot (rb_cap of them): the molecule's cell, the cell's first and end slots, and the
	// molecule's previous slot
	int4* rb_slot = nullptr;
	int64_t rb_cap = 0;
	unsigned long long* builds = nullptr;   // builds so far (device counter)
	// device: bricks of the last build, sparse [0] and dense [1], and the work queues of the sparse [3]
	// and dense [2] list kernels; brick_list: the dense bricks' indices, then (from nbricks on) the
	// sparse ones, in the order the build found them
	unsigned* brick_counts = nullptr;
	int32_t* brick_list = nullptr;
	int* h_sparse = nullptr;                // pinned host copy, read back at the end of each run
	bool lists_valid = false;       // the sort order has not changed since the lists were built
	double* adj = nullptr;          // adjoint buffers: cotangents, outputs, parameter partials
	struct Traj* traj = nullptr;    // device buffers of the trajectory adjoint (traj.cu)
	int64_t adj_cap = 0;
	double* h_scalars = nullptr;    // pinned host mirror
	int* h_status = nullptr;

	// kernel timing
	bool profiling = false;
	cudaEvent_t ev_a[3] = {nullptr, nullptr, nullptr};
	cudaEvent_t ev_b[3] = {nullptr, nullptr, nullptr};
	double prof_ms[3] = {0, 0, 0};
	int64_t prof_count[4] = {0, 0, 0, 0};
};

// Whether the Verlet-skin steps evaluate pruned lists (an inner radius between rc and rc + skin).
inline bool pruning(const Context* c) { return c->skin > 0.0 && c->prune > 0.0 && c->prune < c->skin; }

// ---- launch helpers implemented in the .cu files -------------------------------------------
// Each returns cudaSuccess or the launch error; kernels report data errors in ctx->status.
cudaError_t launch_bin(Context* c, bool permute_forces);
// Verlet-skin mode: wrap, binning on grid g and sort in one cooperative launch that returns at
// once unless *c->rebuild == c->step_id; the sorted arrays end in c->p (buffer roles unchanged)
// and c->perm[i] holds the index before the sort of the molecule now at i. `extra` (nextra planes of
// n doubles, `scratch` as large) are sorted with the molecules. With `always` it builds in every
// launch (the per-step binning of the trajectory adjoint: one launch instead of launch_bin's six).
cudaError_t launch_rebuild(Context* c, const Grid& g, double* extra = nullptr, double* scratch = nullptr,
                           int nextra = 0, bool always = false);
cudaError_t launch_pairs(Context* c);                 // partials -> scalars[0..2] (U6sum, W, npairs)
// The same in the Verlet-skin mode; with kick_mode 1 or 2 the kernels also apply the closing kick
// of the step (mode 2, the last step of a run: forces and velocities stored) or the closing kick,
// the opening kick and drift of the next step into c->q's position arrays (mode 1: the caller swaps
// the position buffers of c->p and c->q afterwards), and write the step record to `record`.
cudaError_t launch_pairs_skin(Context* c, int kick_mode = 0, double dt = 0.0, double* record = nullptr);
int64_t skin_partials_needed(const Context* c);       // reduction partials the skin-mode kernels write
// With skin_check the pre-kick also sets *c->rebuild = c->step_id when a molecule is more than
// skin/2 from its position at the last build.
cudaError_t launch_leapfrog_pre(Context* c, double dt, double vcorr, bool skin_check = false);
// scalars[3] = sum m v^2 (reduced inside the kernel); with a record pointer the kernel also writes
// the step's {Upot, virial, sum m v^2, pairs} there from scalars[0..2].
cudaError_t launch_leapfrog_post(Context* c, double dt_half, double* record = nullptr);
// The closing kick of one step and the opening kick of the next in one pass (mdgpu_run): the same
// operations as launch_leapfrog_post(dt/2) followed by launch_leapfrog_pre(dt, 1).
cudaError_t launch_leapfrog_post_pre(Context* c, double dt, bool skin_check, double* record);
cudaError_t launch_scale(Context* c, double beta);
cudaError_t launch_reduce(Context* c, int64_t nblocks, double* out, int nval);
// Lanes of the adjoint kernel per molecule, and its blocks (of kReduceBlock threads) for n
// molecules: the rows of parameter partials it writes.
constexpr int kAdjLanes = 8;
inline int64_t adjoint_blocks(int64_t n) { return (n * kAdjLanes + kReduceBlock - 1) / kReduceBlock; }
// With `accumulate` the parameter sums are added to pout (otherwise they overwrite it).
cudaError_t launch_adjoint(Context* c, const double* gfx, const double* gfy, const double* gfz, double gU, double* ox,
                           double* oy, double* oz, double* pgrad, double* pout, bool accumulate = false);
// Frees the device buffers of the context's trajectory adjoint (traj.cu).
void free_traj(Context* c);
cudaError_t launch_step_record(Context* c, double* dst);        // dst[0..3] <- step scalars

// Set-up shared by the single-box and the batched contexts (api.cu): LinkedCells geometry of the
// box [0, L), the Comp2Param table, and its device form. Return an MDGPU_* code, message in err.
int setup_grid(const double length[3], double cutoff, double cells_in_cutoff, Grid& g, std::string& err);
// The Verlet-skin grid: an odd cell count of 5 or more in a dimension is lowered by one (cells grow).
void even_grid(Grid& g);
// The grid on which the Verlet-skin lists of radius rc + skin are built (cells of edge >= rc + skin,
// larger in a dilute liquid), from the context's box and loaded positions.
int skin_grid(const Context* c, double skin, Grid& gs, std::string& err);
// Buffers of the cooperative rebuild (launch_rebuild) for the loaded molecules: the build flag, the
// build counter, the barrier and look-back words, the cell counts and the arrival-slot records.
int rebuild_prepare(Context* c);
// Asks for a build in the step c->step_id (sets *c->rebuild on the context's stream).
int request_build(Context* c);
int setup_species(int ncomp, const mdgpu_component* comps, const double* mix, double rc_lj, Species& sp,
                  std::string& err);
PairParams pair_params(const Species& sp, double rc, double rc_lj);

// Status helpers of api.cu for the other entry-point files: read and clear the device status word
// (synchronises the stream) and map it to an MDGPU_* code; record an error message.
int check_device_status(Context* c);
int set_error(Context* c, int code, const std::string& msg);
int set_cuda_error(Context* c, cudaError_t e, const char* where);

// cudaDevAttrMaxSharedMemoryPerBlockOptin of a device, queried once per device (api.cu).
int device_max_optin(int device);

// Timing brackets around a group of launches (0 = binning, 1 = pairs, 2 = integration).
void prof_begin(Context* c, int group);
void prof_end(Context* c, int group, int launches);
void count_launches(Context* c, int launches);

}  // namespace mdgpu

struct mdgpu_ctx {
	mdgpu::Context c;
};
