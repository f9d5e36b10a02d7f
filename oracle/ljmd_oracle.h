/*
 * Plain-C oracle for MarDyn's single-site Lennard-Jones 12-6 hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the parity tests, the package's smoke check
 * and the benchmark's CPU-baseline leg compare against; the product never links or calls it.
 *
 * It restates, sequentially and in the same order of floating-point operations, what the
 * reference does per time step for single-site LJ molecules:
 *   LinkedCells (geometry, binning, neighbour offsets, deleteOuterParticles),
 *   DomainDecompDummy::exchangeMolecules (periodic halo images),
 *   BlockTraverse::traversePairs + ParticlePairs2PotForceAdapter + PotForce/PotForceLJ,
 *   Leapfrog / Molecule::upd_preF / upd_postF, Domain::calculateGlobalValues (Upot, virial, T, beta),
 *   Comp2Param::initialize, Component::addLJcenter, Domain::initFarFieldCorr,
 *   and the RDF pair counting hook (RDF::observeRDF).
 * Each function in ljmd_oracle.c names the reference file:line it follows.
 * The molecule container keeps the reference's std::list order (push_front on insertion),
 * so the summation order -- and hence every bit of F, Upot and the virial -- matches the
 * compiled reference.
 */
#ifndef LJMD_ORACLE_H
#define LJMD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sys orc_sys;

/* Status codes: 0 = ok; the others mirror the reference's exit() paths. */
#define ORC_OK 0
#define ORC_ERR_BOX_TOO_SMALL 5      /* LinkedCells.cpp:81-88 exit(5) */
#define ORC_ERR_SAME_POSITION 11     /* Molecule.cpp:455-456 exit(1) */
#define ORC_ERR_OUTSIDE_HALO 12      /* LinkedCells.cpp:539-541 error message */
#define ORC_ERR_ARGS 13
#define ORC_ERR_EXPLOSION 14         /* Domain.cpp:266-318 selective thermostat (not restated) */

/* ncomp components with one LJ centre each at the origin.
 * mix holds (xi, eta) for i<j in the reference's order (InputOldstyle.cpp:206-215). */
orc_sys* orc_create(const double length[3], double rc, double rcLJ, double cells_in_cutoff, int ncomp,
                    const double* eps, const double* sigma, const double* mass, const int* do_shift,
                    const double* mix);
void orc_destroy(orc_sys* s);
int orc_status(const orc_sys* s);

/* InputOldstyle::readPhaseSpace: addParticle for each molecule in file order. cid is 0-based. */
int orc_add_particles(orc_sys* s, long n, const unsigned long* id, const int* cid, const double* r,
                      const double* v);
/* Tail of Simulation::initConfigOldstyle: far-field correction, update(), deleteOuterParticles(). */
int orc_init(orc_sys* s, double target_temperature, int nve);
/* Simulation::prepare_start: first force evaluation and global values. */
int orc_prepare_start(orc_sys* s);
/* Simulation::simulateStep for one step of length dt; tfactor is Simulation::Tfactor(simstep). */
int orc_step(orc_sys* s, double dt, double tfactor);

long orc_count(const orc_sys* s);
/* Molecules in container order; any pointer may be NULL. cell[] is getCellIndexOfMolecule. */
void orc_get(const orc_sys* s, unsigned long* id, int* cid, double* r, double* v, double* F, long* cell);
/* out[0..12] = local Upot, local virial, summv2 (of Leapfrog::transition2to3), global Upot,
 *              global virial, T, beta_trans, UpotCorr, VirialCorr, number of processPair calls of
 *              the last traversal, sum m v^2 of the molecules at the end of the step, and the
 *              local Upot and virial of the same pair terms summed with compensation (accurate to
 *              ~1e-16 relative, unlike the reference's sequential sums) */
void orc_scalars(const orc_sys* s, double* out);
/* LinkedCells geometry: out_i[0..8] = boxWidthInNumCells[3], haloWidthInNumCells[3], cellsPerDim[3];
 * out_d[0..8] = cellLength[3], haloBoundingBoxMin[3], haloBoundingBoxMax[3] */
void orc_geometry(const orc_sys* s, int* out_i, double* out_d);
/* getCellIndexOfMolecule for an arbitrary position (LinkedCells.cpp:535-551). */
long orc_cell_index(const orc_sys* s, const double r[3]);
/* Comp2Param stream entries for (ci, cj): eps24, sig2, shift6. */
void orc_params(const orc_sys* s, int ci, int cj, double* out3);

/* Pieces of the step, for tests that drive the container like the reference's unit tests do. */
int orc_update(orc_sys* s);                 /* LinkedCells::update */
int orc_exchange(orc_sys* s);               /* DomainDecompDummy::exchangeMolecules */
int orc_traverse(orc_sys* s);               /* LinkedCells::traversePairs (+ calcFM) */
int orc_delete_outer(orc_sys* s);           /* LinkedCells::deleteOuterParticles */
/* RDF::observeRDF: count MOLECULE_MOLECULE pairs with sqrt(dd)/interval binned, until disabled. */
void orc_rdf_enable(orc_sys* s, double interval, int bins);
void orc_rdf_counts(const orc_sys* s, unsigned long* out);

#ifdef __cplusplus
}
#endif
#endif
