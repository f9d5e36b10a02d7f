/*
 * mdgpu.h -- C ABI of the B200 (sm_100a) short-range Lennard-Jones hot path that stands in for
 * MarDyn's LinkedCells container, its LJ pair handler and its Leapfrog integrator.
 *
 * All entry points take plain host pointers and sizes (no CUDA or torch types), return an int
 * status (MDGPU_OK = 0) and leave a message for mdgpu_last_error(). Particle arrays are given and
 * returned in the caller's order (the order of the last mdgpu_set_particles call); positions,
 * velocities and forces are (n, 3) row-major doubles. Component ids are 0-based.
 *
 * Reference interfaces (paths relative to madpac/mardyn/) each entry point replaces are named
 * beside it. A thin C++ shim (a ParticleContainer and an Integrator subclass on the MarDyn side)
 * binds them to MarDyn's simulation loop.
 */
#ifndef MDGPU_H
#define MDGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference's exit() paths become status codes) ---------------------- */
#define MDGPU_OK 0
#define MDGPU_ERR_ARG 1              /* bad argument or unsupported configuration */
#define MDGPU_ERR_CUDA 2             /* a CUDA runtime call failed */
#define MDGPU_ERR_STATE 3            /* cells invalid: call mdgpu_update first (LinkedCells.cpp:294-297 exit(1)) */
#define MDGPU_ERR_BOX_TOO_SMALL 5    /* fewer than 2 cells per dimension (LinkedCells.cpp:81-88 exit(5)) */
#define MDGPU_ERR_OUTSIDE_HALO 6     /* a molecule left the halo box in one step (LinkedCells.cpp:539-541) */
#define MDGPU_ERR_SAME_POSITION 7    /* two molecules at the same position (Molecule.cpp:455-456 exit(1)) */
#define MDGPU_ERR_NONFINITE 8        /* a force, energy or velocity became NaN/Inf */
#define MDGPU_ERR_TIMEOUT 9          /* a bounded device-side wait gave up */
#define MDGPU_ERR_CAPACITY 10        /* a workload exceeds a fixed device buffer */

/* ---- precision modes ---------------------------------------------------------------------- */
#define MDGPU_FP64 0   /* every pair in double precision, same operation order as PotForceLJ */
#define MDGPU_MIXED 1  /* pair arithmetic in FP32, forces/energy/virial accumulated in FP64 */

/* One single-site LJ component: one LJ centre at the molecule origin.
 * Mirrors Component::addLJcenter (molecules/Component.cpp:44-72) with do_shift the
 * TRUNCATED_SHIFTED flag read by InputOldstyle (io/InputOldstyle.cpp:162-166). */
typedef struct mdgpu_component {
	double eps;
	double sigma;
	double mass;
	int do_shift;
} mdgpu_component;

typedef struct mdgpu_ctx mdgpu_ctx;

/* Build a container for a periodic box [0, length) on CUDA device `device`.
 * Replaces the LinkedCells constructor (particleContainer/LinkedCells.cpp:41-94), its
 * initializeCells/calculateNeighbourIndices (:457-533), Comp2Param::initialize
 * (molecules/Comp2Param.cpp:28-115) and Domain::initParameterStreams (Domain.cpp:570-572).
 * cutoff is cutoffRadius (cells and pair search), lj_cutoff is LJCutoffRadius (0 = cutoff);
 * cells_in_cutoff must be 1. mix holds (xi, eta) for each component pair i<j in the order of
 * InputOldstyle.cpp:206-215 (may be NULL for one component). */
int mdgpu_create(mdgpu_ctx** out, const double length[3], double cutoff, double lj_cutoff,
                 double cells_in_cutoff, int ncomp, const mdgpu_component* comps, const double* mix,
                 int precision, int device);
/* Frees every device buffer of the context. */
int mdgpu_destroy(mdgpu_ctx* ctx);
/* Message of the last failed call on this context ("" if none). */
const char* mdgpu_last_error(const mdgpu_ctx* ctx);
/* Switch between MDGPU_FP64 and MDGPU_MIXED. */
int mdgpu_set_precision(mdgpu_ctx* ctx, int precision);

/* Select the pair kernel: 0 = shared-memory brick kernel (default), 1 = simple per-molecule
 * gather kernel (same arithmetic, kept as an independent second implementation). */
int mdgpu_set_pair_kernel(mdgpu_ctx* ctx, int kind);

/* Load n molecules (replaces the InputOldstyle::readPhaseSpace -> LinkedCells::addParticle loop,
 * io/InputOldstyle.cpp:324-378, LinkedCells.cpp:182-204). F may be NULL (zero forces). */
int mdgpu_set_particles(mdgpu_ctx* ctx, int64_t n, const uint64_t* id, const int32_t* cid,
                        const double* r, const double* v, const double* F);
/* Overwrite positions and velocities of the loaded molecules (caller order). */
int mdgpu_set_state(mdgpu_ctx* ctx, int64_t n, const double* r, const double* v);
/* Read molecules back in caller order (replaces iteration with ParticleContainer::begin/next,
 * ParticleContainer.h:100-113). Any output pointer may be NULL. */
int mdgpu_get_particles(mdgpu_ctx* ctx, int64_t n, uint64_t* id, int32_t* cid, double* r, double* v,
                        double* F);
/* Write the loaded molecules as an old-style phase-space file in the layout of the reference's
 * checkpoint (replaces Domain::writeCheckpoint, Domain.cpp:462-568, with
 * DomainDecompDummy::writeMoleculesToFile and Molecule::write, parallel/DomainDecompDummy.cpp:144-154,
 * molecules/Molecule.cpp:263-270): header with currentTime, the box, the target temperature,
 * the components, mixing coefficients and epsilonRF, then one ICRVQD line per molecule in caller
 * order. digits: significant digits of the molecule lines, 0 = the reference's 6 (17 keeps the
 * exact doubles). */
int mdgpu_write_checkpoint(mdgpu_ctx* ctx, const char* path, double current_time, double temperature,
                           double epsilon_rf, int digits);
/* Load the molecules of an old-style phase-space file (replaces InputOldstyle::readPhaseSpaceHeader
 * and readPhaseSpace, io/InputOldstyle.cpp:35-392, feeding LinkedCells::addParticle): formats
 * ICRVQD, ICRVFQDM, ICRV and IRV; the file's box and single-site LJ components must match the
 * context's (MDGPU_ERR_ARG otherwise). current_time and temperature (may be NULL) receive the
 * header's values. */
int mdgpu_read_phase_space(mdgpu_ctx* ctx, const char* path, double* current_time, double* temperature);
/* Number of molecules held (replaces LinkedCells::getNumberOfParticles, LinkedCells.cpp:301-303). */
int mdgpu_num_particles(const mdgpu_ctx* ctx, int64_t* n);
/* Cell geometry: box_cells[3] = boxWidthInNumCells, cell_length[3], halo_min[3]
 * (LinkedCells.cpp:54-66). */
int mdgpu_get_geometry(const mdgpu_ctx* ctx, int32_t box_cells[3], double cell_length[3],
                       double halo_min[3]);

/* Periodic wrap and linked-cell binning by counting sort (replaces LinkedCells::update,
 * LinkedCells.cpp:165-180, together with the wrap that DomainDecompDummy::exchangeMolecules +
 * LinkedCells::deleteOuterParticles perform, parallel/DomainDecompDummy.cpp:22-116,
 * LinkedCells.cpp:339-371). */
int mdgpu_update(mdgpu_ctx* ctx);
/* Cell index of each molecule in caller order, in the reference's halo-inclusive numbering
 * (LinkedCells::getCellIndexOfMolecule, LinkedCells.cpp:535-551). */
int mdgpu_get_cell_index(mdgpu_ctx* ctx, int64_t n, int64_t* cell);
/* Forces on all molecules plus the local potential energy and virial (replaces
 * LinkedCells::traversePairs -> BlockTraverse::traversePairs, BlockTraverse.cpp:89-350, with
 * ParticlePairs2PotForceAdapter::init/processPair/finish, adapter/ParticlePairs2PotForceAdapter.h:52-115,
 * and PotForce/PotForceLJ, molecules/potforce.h:41-53, 319-363). upot and virial receive what
 * finish() stores with Domain::setLocalUpot/setLocalVirial (Domain.cpp:102-108); npairs (may be
 * NULL) receives the number of unordered pairs with r < cutoff. */
int mdgpu_traverse_pairs(mdgpu_ctx* ctx, double* upot, double* virial, double* npairs);
/* Leapfrog first half: v = vcorr*v + dt/(2m)*F; r += dt*v for every molecule (replaces
 * Leapfrog::transition1to2, integrators/Leapfrog.cpp:37-51, Molecule::upd_preF, Molecule.cpp:128-135). */
int mdgpu_leapfrog_pre(mdgpu_ctx* ctx, double dt, double vcorr);
/* Leapfrog second half: v += dt_half/m*F and sum m v^2 (replaces Leapfrog::transition2to3,
 * Leapfrog.cpp:53-99, Molecule::upd_postF, Molecule.cpp:193-216). */
int mdgpu_leapfrog_post(mdgpu_ctx* ctx, double dt_half, double* summv2);
/* v *= beta for every molecule (the velocity scaling of Simulation::thermostatEtc,
 * Simulation.cpp:1172-1176). */
int mdgpu_scale_velocities(mdgpu_ctx* ctx, double beta);
/* Far-field LJ corrections UpotCorr and VirialCorr for unshifted pairs (replaces
 * Domain::initFarFieldCorr, Domain.cpp:574-677, single-centre LJ part). */
int mdgpu_far_field_correction(mdgpu_ctx* ctx, double* upot_corr, double* virial_corr);
/* One NVE/thermostatted time step as Simulation::simulateStep runs it (Simulation.cpp:1218-1229):
 * leapfrog_pre(dt, vcorr), update, traverse_pairs, leapfrog_post(dt/2). out[0..3] = local Upot,
 * local virial, sum m v^2, pair count. */
int mdgpu_step(mdgpu_ctx* ctx, double dt, double vcorr, double* out4);
/* nsteps NVE steps without host round trips; per_step (may be NULL) receives nsteps rows of the
 * four values of mdgpu_step. */
int mdgpu_run(mdgpu_ctx* ctx, int32_t nsteps, double dt, double* per_step);

/* Enqueue nsteps NVE steps on the context's stream and return without waiting; each step's four
 * values (see mdgpu_step) are appended to a device-side record kept until mdgpu_read_steps. */
int mdgpu_run_async(mdgpu_ctx* ctx, int32_t nsteps, double dt);
/* Wait for the enqueued steps, copy the first nsteps records (nsteps x 4), clear the record and
 * report status. */
int mdgpu_read_steps(mdgpu_ctx* ctx, int32_t nsteps, double* per_step);

/* Adjoint of the forces and potential energy at the current positions (call after mdgpu_update;
 * no counterpart in the reference, which has no gradients). Given the cotangents gF = dL/dF
 * ((n, 3), caller order) and gU = dL/dUpot of a loss L, returns dL/dr ((n, 3), caller order) and,
 * for every component pair (a, b), dL/d(eps_ab) and dL/d(sigma_ab) in ncomp x ncomp symmetric
 * arrays (may be NULL), where eps_ab = eps24/24 and sigma_ab = sqrt(sig2) of the Comp2Param stream
 * (molecules/Comp2Param.cpp:28-115) and truncated-shifted pairs include the shift's dependence.
 * Double precision. */
int mdgpu_adjoint(mdgpu_ctx* ctx, const double* gF, double gU, double* dL_dr, double* dL_deps, double* dL_dsigma);

/* Reverse-mode gradient through an NVE Leapfrog trajectory on the device (no counterpart in the
 * reference). mdgpu_traj_forward runs nsteps steps of Simulation::simulateStep with the per-step
 * binning (skin 0; Leapfrog vcorr = 1) from the loaded state, keeping (r, v) every
 * checkpoint_every steps in device memory, and leaves the final state in the context (upot_final:
 * its local Upot). mdgpu_traj_backward takes the cotangents gF ((n, 3), caller order) and gU of
 * the final forces and Upot and returns dL/dr_0 and dL/dv_0 ((n, 3), caller order; dL_dv0 may be
 * NULL) and the ncomp x ncomp gradients with respect to eps_ab and sigma_ab (as mdgpu_adjoint
 * reports them; either may be NULL), recomputing each segment from its snapshot on the device
 * (recomputed_steps, may be NULL, receives how many steps that took); afterwards the context holds
 * the start state again. Arithmetic in the context's precision (the mixed form: FP32 pair terms,
 * FP64 sums). */
int mdgpu_traj_forward(mdgpu_ctx* ctx, int32_t nsteps, int32_t checkpoint_every, double dt, double* upot_final);
int mdgpu_traj_backward(mdgpu_ctx* ctx, const double* gF, double gU, double* dL_dr0, double* dL_dv0,
                        double* dL_deps, double* dL_dsigma, int64_t* recomputed_steps);
/* Device time (CUDA events on the context's stream) of the adjoint-kernel launches of the last
 * mdgpu_traj_backward that ran with mdgpu_profile_enable on, and how many there were. */
int mdgpu_traj_adjoint_time(mdgpu_ctx* ctx, double* ms, int64_t* launches);

/* ---- molecule-side operations of MaDPaC's coupled step --------------------------------------
 * MarDynSimulation::simulateStep (coupling/MarDynSimulation.cpp:61-160) interleaves the MD step with
 * the lattice-Boltzmann connector's operations on molecules; these are the molecule-side ones on the
 * device container (per-step binning, skin 0), the connector's parameters given as arguments.
 *
 * mdgpu_reflect_boundary replaces ReflectingBoundary::applyBoundary (coupling/boundary/
 * ReflectingBoundary.cpp:47-130); call it after mdgpu_leapfrog_pre and before mdgpu_update. Each
 * molecule outside the box in a dimension i < dim (2 or 3) has v_i negated and is moved back inside
 * with the reference's arithmetic (r + (-r - 2r) at the lower face, r - 2 (r - L) at the upper one),
 * except beyond the upper face of stream_out_dir when the stream-out is on (always without a moving
 * wall, as the reference sets it): those are counted in *streamed_out (may be NULL) and left as they
 * are (the connector deletes them; the device container's next mdgpu_update would wrap them). */
int mdgpu_reflect_boundary(mdgpu_ctx* ctx, int32_t dim, int32_t stream_out_dir, int32_t moving_wall, int32_t stream_out,
                           int64_t* streamed_out);
/* The wall force of ForceBoundary::applyBoundary (coupling/boundary/ForceBoundary.cpp:52-226) added to
 * the forces of the molecules within `border` of a face (X, Y, and Z when dim is 3; [0, border) and
 * [L - border, L), the box in the other dimensions): ForceBoundary::calcFm's piecewise fit
 * (ForceBoundary.h:56-82) of the distance to the face, outward at the upper faces and scaled by
 * stream_damping at the upper face of stream_out_dir. Call it after mdgpu_traverse_pairs. (In the
 * reference the region lists are filled in copies -- FBoundary::getLower/getUpper take them by
 * value -- so its applyBoundary changes no force; this is the force its code computes.) */
int mdgpu_force_boundary(mdgpu_ctx* ctx, int32_t dim, double border, int32_t stream_out_dir, double stream_damping);

/* The coupling-cell grid of the connector's DataContainer (madpac/core/DataContainer.cpp:209-261):
 * molecules at lower <= r <= upper (first dim dimensions) belong to cell
 * ((ix * size[1] + iy) * size[2] + iz), ix = (int) ((x - lower[0]) / cell_size); size[2] = 1 in 2D. */
typedef struct mdgpu_coupling_cells {
	double lower[3];
	double upper[3];
	double cell_size;
	int32_t size[3];
	int32_t dim;
} mdgpu_coupling_cells;

typedef struct mdgpu_thermostat mdgpu_thermostat;
/* CellWiseThermostat (coupling/thermostat/CellWiseThermostat.cpp:46-156) on the device container:
 * mdgpu_thermostat_apply(th, iteration) after mdgpu_leapfrog_post does applyThermostat(iteration):
 * each call adds every molecule's velocity to its coupling cell's sums; when iteration is a multiple
 * of `interval` it forms the cells' mean velocities in the directed dimensions, their peculiar
 * kinetic energies E and rescales v = (v - vc)(1 + gamma (beta - 1)) + vc with
 * beta = sqrt(1.5 samples / interval * T / E), then clears the sums. The global-energy diagnostics
 * of updateGlobalE do not act on molecules and are not computed. The per-cell sums are 64-bit fixed
 * point in steps of 2^-40 (independent of the order of the additions); a cell whose velocity or
 * kinetic-energy sum reaches 2^23 makes the call fail with MDGPU_ERR_CAPACITY. */
int mdgpu_thermostat_create(mdgpu_thermostat** out, mdgpu_ctx* ctx, const mdgpu_coupling_cells* cells,
                            double target_temperature, double gamma, int32_t interval, const int32_t directed[3]);
int mdgpu_thermostat_apply(mdgpu_thermostat* th, int64_t iteration);
int mdgpu_thermostat_destroy(mdgpu_thermostat* th);

/* Device-side timing of the kernels this context launches, for benchmarking: when enabled, CUDA
 * events on the context's stream bracket the binning, pair and integration kernels. times_ms[0..2]
 * = total binning, pair, integration milliseconds since the last reset; counts[0..3] = launches of
 * each group and of all kernels. */
int mdgpu_profile_enable(mdgpu_ctx* ctx, int enable);
int mdgpu_profile_read(mdgpu_ctx* ctx, double times_ms[3], int64_t counts[4], int reset);
/* The cudaStream_t the context launches on, as an opaque pointer. */
int mdgpu_get_stream(const mdgpu_ctx* ctx, void** stream);
/* Block until the context's stream is idle and report any pending device status. */
int mdgpu_synchronize(mdgpu_ctx* ctx);
/* Measured peak FMA throughput of CUDA device `device` (dependent FMA chains in registers, all
 * SMs busy), in TFLOP/s counting an FMA as 2 flops; used as the roofline of the pair kernels. */
int mdgpu_device_peaks(int device, double* fp32_tflops, double* fp64_tflops);

/* Forces, local potential energy and virial of one periodic box without any device allocation.
 * No counterpart in the reference: this is for callers that cannot call cudaMalloc while they
 * run (hosts that own all device memory through their own pool, latency-bound loops that must not
 * block on the driver's allocator). Inputs and outputs are the
 * caller's device buffers: d_r (n, 3) positions and d_cid (n) 0-based component ids in, d_F
 * (n, 3) forces out; upot and virial (host, may be NULL) receive what mdgpu_traverse_pairs
 * returns. All intermediate buffers live in one static device array of about 7.5 MB that every
 * GPU loading the library holds until exit, so n <= 32768 and the cell grid <= 32768 cells
 * (larger inputs return MDGPU_ERR_CAPACITY). Calls share that array and keep its last contents
 * (each call clears what must start at zero); calls that overlap on the GPU race and must be
 * serialised. The first call on a device looks up the array's address with that device current;
 * make it before any stream capture, and do not use the library across a cudaDeviceReset. stream
 * may be NULL (default stream); the call is synchronous: it uploads its parameter table from host
 * memory, waits for the stream and returns upot, virial and the status on the host. The caller's
 * current device is unchanged on return. lj_cutoff 0 means the cutoff; negative values are
 * rejected. errbuf (may be NULL) receives a message of at most errlen bytes. */
int mdgpu_forces_noalloc(int device, void* stream, int64_t n, const double* d_r, const int32_t* d_cid,
                         const double length[3], double cutoff, double lj_cutoff, int ncomp,
                         const mdgpu_component* comps, const double* mix, int precision, double* d_F,
                         double* upot, double* virial, char* errbuf, int errlen);

/* Verlet-skin mode of mdgpu_step / mdgpu_run / mdgpu_run_async (skin > 0; 0 = off, the default).
 * No reference counterpart: the reference rebuilds its cells every step (LinkedCells::update).
 * With a skin, the binning (on cells of edge >= cutoff + skin) and the candidate search run only
 * in steps where some molecule has moved more than skin/2 since the last build, decided on the
 * device; the other steps evaluate each molecule's recorded candidates. Every pair within the
 * cutoff is still evaluated with the exact test (r^2 < rc^2), so forces, Upot and virial are those
 * of the per-step traversal up to summation order. Positions are wrapped into [0, L) at each build
 * and on output (mdgpu_get_particles). After such steps the cell structure is not the reference's:
 * call mdgpu_update before mdgpu_traverse_pairs, mdgpu_get_cell_index or mdgpu_adjoint. */
int mdgpu_set_skin(mdgpu_ctx* ctx, double skin);
/* Number of list builds of the Verlet-skin mode so far (synchronises the context's stream). */
int mdgpu_skin_builds(mdgpu_ctx* ctx, int64_t* builds);
/* Pruned lists of the Verlet-skin mode (0 < prune < skin; 0 = off, the default). No reference
 * counterpart. The steps evaluate inner lists: the entries of each build list that were within
 * cutoff + prune at the last prune. A prune re-filters the build lists at the current positions.
 * It runs after every build, and whenever the per-step largest drifts summed since the last prune
 * reach prune/2, decided on the device. A pair left out of an inner list is therefore beyond the
 * cutoff until the next prune: the same pairs are evaluated as without pruning, fewer entries are
 * read. prune must be in [0, cutoff); it is in effect while it is also below the skin.
 * mdgpu_list_prunes: prunes so far (synchronises the context's stream). */
int mdgpu_set_list_prune(mdgpu_ctx* ctx, double prune);
int mdgpu_list_prunes(mdgpu_ctx* ctx, int64_t* prunes);

/* ---- batched ensemble of independent boxes ------------------------------------------------
 * No reference counterpart: in MarDyn every box is its own Simulation with its own LinkedCells
 * (Simulation.cpp:907-1308), run one after the other. A batch holds nboxes independent periodic
 * boxes [0, L_b) of n_b molecules that share the cutoffs, the components and the precision mode,
 * and advances all of them with one persistent (cooperative) kernel launch per step, replayed from
 * a captured CUDA graph. Per box and step the kernel does what mdgpu_step does for one box
 * (Leapfrog pre, wrap and binning, pair forces, Leapfrog post), with the same arithmetic.
 * Molecule arrays are box-major: box 0's n_0 molecules, then box 1's, and so on. Per-box records
 * are 4 doubles {Upot, virial, sum m v^2, pairs}, as the out4 of mdgpu_step. */
typedef struct mdgpu_batch mdgpu_batch;

/* lengths: nboxes x 3; counts: molecules per box. Boxes whose cell sort does not fit in shared
 * memory (about 17,000 molecules) are rejected with MDGPU_ERR_CAPACITY. */
int mdgpu_batch_create(mdgpu_batch** out, int32_t nboxes, const double* lengths, const int64_t* counts,
                       double cutoff, double lj_cutoff, double cells_in_cutoff, int ncomp,
                       const mdgpu_component* comps, const double* mix, int precision, int device);
int mdgpu_batch_destroy(mdgpu_batch* b);
const char* mdgpu_batch_last_error(const mdgpu_batch* b);
int mdgpu_batch_set_particles(mdgpu_batch* b, int64_t ntotal, const uint64_t* id, const int32_t* cid,
                              const double* r, const double* v);
int mdgpu_batch_get_particles(mdgpu_batch* b, int64_t ntotal, uint64_t* id, int32_t* cid, double* r,
                              double* v, double* F);
/* Initial binning and force evaluation of every box (as Simulation::prepare_start); out: nboxes x 4
 * (may be NULL). */
int mdgpu_batch_prepare(mdgpu_batch* b, double* out);
/* nsteps NVE steps of every box; per_step: nsteps x nboxes x 4 (may be NULL). */
int mdgpu_batch_run(mdgpu_batch* b, int32_t nsteps, double dt, double* per_step);
/* Tile shape of the persistent kernel: per-lane candidate list depth (32 or 64), CTAs per SM
 * (1 or 2; sets the shared-memory staging capacity), brick distribution (0 static, 1 queue). */
int mdgpu_batch_set_tiles(mdgpu_batch* b, int32_t list_cap, int32_t ctas_per_sm, int32_t dynamic);
int mdgpu_batch_get_tiles(const mdgpu_batch* b, int32_t tiles[3]);
/* Times every tile shape for trial_steps steps from the current state (restored afterwards), keeps
 * the fastest; best: its 3 values, ms: device ms per step of each of the 8 candidates (may be NULL),
 * -1 for a candidate not timed: a shape whose staging does not fit, and in the Verlet-skin mode the
 * list depth other than the current one (the depth does not act on skin-mode lists). */
int mdgpu_batch_autotune(mdgpu_batch* b, double dt, int32_t trial_steps, int32_t best[3], double* ms);
/* Device time of the last mdgpu_batch_run (CUDA events around the graph launch). */
int mdgpu_batch_last_run_ms(const mdgpu_batch* b, double* ms);
/* Limit of each grid-barrier wait in nanoseconds (default 2e9); a wait that runs out sets
 * MDGPU_ERR_TIMEOUT and the kernel returns. */
int mdgpu_batch_set_barrier_timeout(mdgpu_batch* b, int64_t ns);
/* Verlet-skin mode of the batch (as mdgpu_set_skin, per box: a box is re-binned and its candidate
 * lists rebuilt inside the step when one of its molecules moved more than skin/2). Takes effect at
 * the next mdgpu_batch_prepare; 0 = off. mdgpu_batch_skin_builds: box list builds so far. */
int mdgpu_batch_set_skin(mdgpu_batch* b, double skin);
int mdgpu_batch_skin_builds(const mdgpu_batch* b, int64_t* builds);

/* ---- rigid multi-centre LJ molecules ------------------------------------------------------
 * Molecules of several LJ centres with orientation q (quaternion w, x, y, z), angular momentum D
 * (space frame) and torque M. Replaces, for such components, the same LinkedCells / pair handler /
 * Leapfrog sequence as the single-centre context: PotForce's loop over centre pairs
 * (molecules/potforce.h:319-363), Molecule::upd_cache and calcFM (molecules/Molecule.cpp:161-190,
 * 386-411), and the rotational half of Molecule::upd_preF / upd_postF (Molecule.cpp:128-159,
 * 193-216). Arrays in the caller's order: r, v, F, D, M are (n, 3), q is (n, 4). */
#define MDGPU_MAX_SITES 6         /* LJ centres + charges per component */
#define MDGPU_MAX_SITE_TOTAL 16   /* LJ centres + charges over all components */

/* One LJ centre at r (principal-axes frame, the origin at the centre of mass), as read by
 * InputOldstyle (io/InputOldstyle.cpp:162-166) and added by Component::addLJcenter
 * (molecules/Component.cpp:44-72); the shift uses LJCutoffRadius as the centre's cutoff. */
typedef struct mdgpu_site {
	double r[3];
	double mass;
	double eps;
	double sigma;
	int do_shift;
} mdgpu_site;

/* A point charge q at r with its mass (Component::addCharge, molecules/Component.cpp:115-133, read by
 * InputOldstyle.cpp:167-171). Charge pairs of molecules within the cutoff interact by the plain
 * Coulomb term of PotForce2Charge (molecules/potforce.h:244-253, 372-386), 4 pi eps0 = 1. */
typedef struct mdgpu_charge {
	double r[3];
	double mass;
	double q;
} mdgpu_charge;

/* A massless point dipole (strength |my|) or linear quadrupole (|Q|) at r with orientation e in the
 * body frame, used as given (Component::addDipole/addQuadrupole, molecules/Component.cpp:135-145,
 * read by InputOldstyle.cpp:172-181). */
typedef struct mdgpu_oriented {
	double r[3];
	double e[3];
	double strength;
} mdgpu_oriented;

typedef struct mdgpu_rigid mdgpu_rigid;

/* nsites[c] LJ centres (at least one) for each component c, listed one component after another in
 * `sites`; ncharges[c] point charges in `charges` the same way (both may be NULL for none);
 * MDGPU_MAX_SITES bounds centres + charges per component. inertia: 3 per component or NULL, values
 * > 0 replace the principal moments computed from the centres and charges (the header's inertia
 * line, InputOldstyle.cpp:188-195). Other arguments as mdgpu_create. On failure *out may still be
 * set (read mdgpu_rigid_last_error, then destroy it). */
int mdgpu_rigid_create(mdgpu_rigid** out, const double length[3], double cutoff, double lj_cutoff,
                       double cells_in_cutoff, int ncomp, const int32_t* nsites, const mdgpu_site* sites,
                       const int32_t* ncharges, const mdgpu_charge* charges, const double* inertia,
                       const double* mix, int precision, int device);
int mdgpu_rigid_destroy(mdgpu_rigid* h);
const char* mdgpu_rigid_last_error(const mdgpu_rigid* h);
int mdgpu_rigid_set_precision(mdgpu_rigid* h, int precision);
/* Point dipoles and quadrupoles of the components (ndipoles[c] and nquadrupoles[c] per component,
 * listed one component after another; either may be NULL) and the reaction field's permittivity
 * epsilon_rf (the header's epsilonRF; 1e10 by default). Call before mdgpu_rigid_set_particles.
 * Every point-polarity pair of molecules within the cutoff then interacts as in PotForce
 * (molecules/potforce.h:65-311, 365-542): charge-quadrupole, charge-dipole, dipole-dipole with the
 * reaction-field term MyRF, dipole-quadrupole and quadrupole-quadrupole, with their direct torques;
 * Upot gains UpotXpoles + MyRF and the virial 3 MyRF (ParticlePairs2PotForceAdapter::finish). The
 * pairs with a dipole or quadrupole are evaluated in double in both precision modes. */
int mdgpu_rigid_set_polarities(mdgpu_rigid* h, const int32_t* ndipoles, const mdgpu_oriented* dipoles,
                               const int32_t* nquadrupoles, const mdgpu_oriented* quadrupoles, double epsilon_rf);
/* The far-field corrections of Domain::initFarFieldCorr (Domain.cpp:574-677) for rigid components:
 * the LJ tail beyond LJCutoffRadius of every unshifted centre pair (TICC/TICS/TISS integrals of
 * CutoffCorrections.cpp over the centres' distances from the centre of mass; MDGPU_ERR_ARG when two
 * of them reach the cutoff together) and the reaction field's self term of each molecule's dipole
 * (its charges' q r plus its dipoles). Host arithmetic only (no context, no device): components as
 * for mdgpu_rigid_create (dipoles as for mdgpu_rigid_set_polarities; NULL for none), counts[c]
 * molecules of component c in the box of edges `length`; lj_cutoff 0 means the cutoff. upot_corr and
 * virial_corr receive the reference's _UpotCorr and _VirialCorr. Negative counts, a dipole direction
 * of zero length, an empty box and a too small LJ cutoff return MDGPU_ERR_ARG; errbuf (may be NULL)
 * receives a message of at most errlen bytes. */
int mdgpu_rigid_far_field_correction(int ncomp, const int32_t* nsites, const mdgpu_site* sites,
                                     const int32_t* ncharges, const mdgpu_charge* charges,
                                     const int32_t* ndipoles, const mdgpu_oriented* dipoles, const double* mix,
                                     const int64_t* counts, const double length[3], double cutoff,
                                     double lj_cutoff, double epsilon_rf, double* upot_corr, double* virial_corr,
                                     char* errbuf, int errlen);
/* Total mass and principal moments of component comp (Component::m, I11/I22/I33). */
int mdgpu_rigid_get_inertia(const mdgpu_rigid* h, int32_t comp, double* mass, double I[3]);
/* Loads the molecules (q and D required); forces and torques start at zero. */
int mdgpu_rigid_set_particles(mdgpu_rigid* h, int64_t n, const uint64_t* id, const int32_t* cid, const double* r,
                              const double* v, const double* q, const double* D);
/* Any output pointer may be NULL. */
int mdgpu_rigid_get_particles(mdgpu_rigid* h, int64_t n, uint64_t* id, int32_t* cid, double* r, double* v, double* F,
                              double* q, double* D, double* M);
/* LinkedCells::update of the molecule centres (with the periodic wrap). */
int mdgpu_rigid_update(mdgpu_rigid* h);
/* Molecule::upd_cache for all molecules, LinkedCells::traversePairs with the LJ centre loop and the
 * charge pairs, and Molecule::calcFM: F and M of every molecule, Upot = Upot6LJ/6 + UpotXpoles
 * (ParticlePairs2PotForceAdapter::finish), the virial sum drm.f and the number of molecule pairs
 * within the cutoff. */
int mdgpu_rigid_traverse_pairs(mdgpu_rigid* h, double* upot, double* virial, double* npairs);
/* Molecule::upd_preF(dt, vcorr, Dcorr) for all molecules (Leapfrog::transition1to2). */
int mdgpu_rigid_leapfrog_pre(mdgpu_rigid* h, double dt, double vcorr, double Dcorr);
/* Molecule::upd_postF(dt_half) for all molecules (Leapfrog::transition2to3): sum m v^2, sum I w^2. */
int mdgpu_rigid_leapfrog_post(mdgpu_rigid* h, double dt_half, double* summv2, double* sum_iw2);
/* nsteps NVE steps of Simulation::simulateStep (after the forces of the start are in place);
 * per_step (may be NULL): 5 doubles per step {Upot, virial, sum m v^2, sum I w^2, pairs}. */
int mdgpu_rigid_run(mdgpu_rigid* h, int32_t nsteps, double dt, double* per_step);
/* Verlet-skin mode of mdgpu_rigid_run (no reference counterpart; skin 0 turns it off): each step
 * tests every molecule pair of a list of radius rc + skin with the exact cutoff, and the rebinning
 * (on cells of edge >= rc + skin) and the list build run only when a molecule has moved more than
 * skin/2 since the last build; 0 < skin <= rc/2. list_cap: list entries per molecule (0: from the
 * densest cell of the loaded positions); a molecule with more candidates scans its cells instead.
 * After skin steps the cells are not the reference's: mdgpu_rigid_traverse_pairs needs
 * mdgpu_rigid_update first. */
int mdgpu_rigid_set_skin(mdgpu_rigid* h, double skin, int32_t list_cap);
/* List builds of the rigid context's skin mode so far (synchronises its stream). */
int mdgpu_rigid_skin_builds(mdgpu_rigid* h, int64_t* builds);
int mdgpu_rigid_get_stream(const mdgpu_rigid* h, void** stream);
/* Kernel timing of the context, as mdgpu_profile_enable / mdgpu_profile_read (groups: binning,
 * site rotation + pairs, integration; counts[3] = all launches so far). */
int mdgpu_rigid_profile_enable(mdgpu_rigid* h, int enable);
int mdgpu_rigid_profile_read(mdgpu_rigid* h, double times_ms[3], int64_t counts[4], int reset);

#ifdef __cplusplus
}
#endif
#endif /* MDGPU_H */
