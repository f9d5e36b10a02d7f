/*
 * Plain-C oracle for MarDyn's single-site LJ 12-6 hot path.  TEST INFRASTRUCTURE ONLY:
 * the tests, the package's smoke check and the benchmark's CPU-baseline leg use it as the
 * checker; the product never links or calls it.  See ljmd_oracle.h for the scope.
 *
 * Reference paths below are relative to the MarDyn source tree (madpac/mardyn/).
 * Compile without floating-point contraction (-ffp-contract=off) so that every double
 * operation rounds exactly as in the reference build (x86-64 g++ -O3, no FMA).
 */
#include "ljmd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
	unsigned long id;
	int cid;
	double r[3], v[3], F[3];
} orc_mol;

typedef struct {
	long* item;
	long n, cap;
} orc_cell;

struct orc_sys {
	int status;
	/* Domain / container configuration */
	double L[3];
	double rc, rcLJ, cic;
	int ncomp;
	double *eps24, *sig2, *shift6; /* ncomp*ncomp, Comp2Param stream entries */
	double* mass;                  /* per component */
	double *eps, *sigma;
	int* do_shift;
	/* LinkedCells geometry (LinkedCells.h:282-290) */
	int boxw[3], halow[3], cpd[3];
	double cellLength[3], haloLength[3], haloMin[3], haloMax[3];
	long ncells;
	char* region; /* 0 halo, 1 boundary, 2 inner */
	long *inner, *boundary, *halo;
	long ninner, nboundary, nhalo;
	long fwd[512], bwd[512];
	int nfwd, nbwd;
	orc_cell* cells;
	int cells_valid;
	/* the std::list<Molecule>: a pool plus the list order; the list grows at its front */
	orc_mol* pool;
	long pool_n, pool_cap;
	long* order_buf;
	long head, tail, order_cap;
	/* Domain values */
	double local_upot, local_virial, summv2, summv2_end;
	double upot_corr, virial_corr;
	double global_upot, global_virial, T, beta_trans, T_target;
	int nve;
	double npairs;
	double u6_hi, u6_lo, w_hi, w_lo; /* compensated sums of the same pair terms */
	/* RDF */
	int rdf_on, rdf_bins;
	double rdf_interval, rdf_max2;
	unsigned long* rdf_counts;
};

/* ---------------------------------------------------------------- helpers */

static void cell_push(orc_cell* c, long idx) {
	if (c->n == c->cap) {
		c->cap = c->cap ? 2 * c->cap : 8;
		c->item = (long*) realloc(c->item, (size_t) c->cap * sizeof(long));
	}
	c->item[c->n++] = idx;
}

static long pool_new(orc_sys* s) {
	if (s->pool_n == s->pool_cap) {
		s->pool_cap = s->pool_cap ? 2 * s->pool_cap : 1024;
		s->pool = (orc_mol*) realloc(s->pool, (size_t) s->pool_cap * sizeof(orc_mol));
	}
	return s->pool_n++;
}

/* std::list::push_front: the order buffer keeps free room in front of head. */
static void list_push_front(orc_sys* s, long idx) {
	if (s->head == 0) {
		long n = s->tail - s->head;
		long cap = 2 * s->order_cap + 1024;
		long* nb = (long*) malloc((size_t) cap * sizeof(long));
		long nh = cap - n - 16;
		memcpy(nb + nh, s->order_buf + s->head, (size_t) n * sizeof(long));
		free(s->order_buf);
		s->order_buf = nb;
		s->order_cap = cap;
		s->head = nh;
		s->tail = nh + n;
	}
	s->order_buf[--s->head] = idx;
}

/* LinkedCells::cellIndexOf3DIndex, LinkedCells.cpp:549-551 */
static long cell_index_3d(const orc_sys* s, int x, int y, int z) {
	return ((long) z * s->cpd[1] + y) * s->cpd[0] + x;
}

/* LinkedCells::getCellIndexOfMolecule, LinkedCells.cpp:535-547 */
long orc_cell_index(const orc_sys* s, const double r[3]) {
	int ci[3];
	for (int d = 0; d < 3; d++) ci[d] = (int) floor((r[d] - s->haloMin[d]) / s->cellLength[d]);
	return cell_index_3d(s, ci[0], ci[1], ci[2]);
}

static int in_halo_box(const orc_sys* s, const double r[3]) {
	for (int d = 0; d < 3; d++)
		if (!(r[d] >= s->haloMin[d] && r[d] < s->haloMax[d])) return 0;
	return 1;
}

/* ---------------------------------------------------------------- setup */

/* Component::addLJcenter shift (Component.cpp:44-55) and Comp2Param::initialize
 * (Comp2Param.cpp:28-115) for one LJ centre per component. */
static void init_params(orc_sys* s, const double* mix) {
	int n = s->ncomp;
	int mixpos = 0;
	for (int i = 0; i < n; i++) {
		/* same-component stream entry; shift6 is the centre's own (Component.cpp:47-55) */
		double shift6i = 0.0;
		if (s->do_shift[i]) {
			double sigperrc2 = s->sigma[i] * s->sigma[i] / (s->rcLJ * s->rcLJ);
			double sigperrc6 = sigperrc2 * sigperrc2 * sigperrc2;
			shift6i = 24.0 * s->eps[i] * (sigperrc6 - sigperrc6 * sigperrc6);
		}
		double e24 = 24. * sqrt(s->eps[i] * s->eps[i]);
		double sg = .5 * (s->sigma[i] + s->sigma[i]);
		sg *= sg;
		s->eps24[i * n + i] = e24;
		s->sig2[i * n + i] = sg;
		s->shift6[i * n + i] = shift6i;
		for (int j = i + 1; j < n; j++) {
			double xi = mix[mixpos++];
			double eta = mix[mixpos++];
			/* (i, j) stream, Comp2Param.cpp:72-92 */
			double epsilon24 = 24. * xi * sqrt(s->eps[i] * s->eps[j]);
			double sigma2 = eta * .5 * (s->sigma[i] + s->sigma[j]);
			sigma2 *= sigma2;
			double sigperrc2 = sigma2 / (s->rcLJ * s->rcLJ);
			double sigperrc6 = sigperrc2 * sigperrc2 * sigperrc2;
			double sh = epsilon24 * (sigperrc6 - sigperrc6 * sigperrc6);
			s->eps24[i * n + j] = epsilon24;
			s->sig2[i * n + j] = sigma2;
			s->shift6[i * n + j] = sh;
			/* (j, i) stream, Comp2Param.cpp:94-113 */
			epsilon24 = 24. * xi * sqrt(s->eps[j] * s->eps[i]);
			sigma2 = eta * .5 * (s->sigma[j] + s->sigma[i]);
			sigma2 *= sigma2;
			sigperrc2 = sigma2 / (s->rcLJ * s->rcLJ);
			sigperrc6 = sigperrc2 * sigperrc2 * sigperrc2;
			sh = epsilon24 * (sigperrc6 - sigperrc6 * sigperrc6);
			s->eps24[j * n + i] = epsilon24;
			s->sig2[j * n + i] = sigma2;
			s->shift6[j * n + i] = sh;
		}
	}
}

/* LinkedCells constructor geometry (LinkedCells.cpp:54-88), initializeCells (:457-487),
 * calculateNeighbourIndices (:489-533). Bounding box is [0, L) (DomainDecompDummy.cpp:137-142). */
static int init_cells(orc_sys* s) {
	long ncells = 1;
	for (int d = 0; d < 3; d++) {
		double bbmin = 0.0, bbmax = s->L[d];
		s->boxw[d] = (int) floor((bbmax - bbmin) / s->rc * s->cic);
		if (s->boxw[d] == 0) s->boxw[d] = 1;
		s->cellLength[d] = (bbmax - bbmin) / s->boxw[d];
		s->halow[d] = (int) ceil(s->cic);
		s->haloLength[d] = s->halow[d] * s->cellLength[d];
		s->haloMin[d] = bbmin - s->haloLength[d];
		s->haloMax[d] = bbmax + s->haloLength[d];
		s->cpd[d] = s->boxw[d] + 2 * s->halow[d];
		ncells *= s->cpd[d];
	}
	for (int d = 0; d < 3; d++)
		if (s->boxw[d] < s->halow[d]) return ORC_ERR_BOX_TOO_SMALL;
	s->ncells = ncells;
	s->cells = (orc_cell*) calloc((size_t) ncells, sizeof(orc_cell));
	s->region = (char*) calloc((size_t) ncells, 1);
	s->inner = (long*) malloc((size_t) ncells * sizeof(long));
	s->boundary = (long*) malloc((size_t) ncells * sizeof(long));
	s->halo = (long*) malloc((size_t) ncells * sizeof(long));
	s->ninner = s->nboundary = s->nhalo = 0;
	for (int iz = 0; iz < s->cpd[2]; ++iz)
		for (int iy = 0; iy < s->cpd[1]; ++iy)
			for (int ix = 0; ix < s->cpd[0]; ++ix) {
				long ci = cell_index_3d(s, ix, iy, iz);
				const int* hw = s->halow;
				const int* cp = s->cpd;
				if (ix < hw[0] || iy < hw[1] || iz < hw[2] || ix >= cp[0] - hw[0] || iy >= cp[1] - hw[1] ||
				    iz >= cp[2] - hw[2]) {
					s->region[ci] = 0;
					s->halo[s->nhalo++] = ci;
				} else if (ix < 2 * hw[0] || iy < 2 * hw[1] || iz < 2 * hw[2] || ix >= cp[0] - 2 * hw[0] ||
				           iy >= cp[1] - 2 * hw[1] || iz >= cp[2] - 2 * hw[2]) {
					s->region[ci] = 1;
					s->boundary[s->nboundary++] = ci;
				} else {
					s->region[ci] = 2;
					s->inner[s->ninner++] = ci;
				}
			}
	s->nfwd = s->nbwd = 0;
	double rc2 = pow(s->rc, 2);
	for (int z = -s->halow[2]; z <= s->halow[2]; z++) {
		double zd2 = z != 0 ? pow((abs(z) - 1) * s->cellLength[2], 2) : 0;
		for (int y = -s->halow[1]; y <= s->halow[1]; y++) {
			double yd2 = y != 0 ? pow((abs(y) - 1) * s->cellLength[1], 2) : 0;
			for (int x = -s->halow[0]; x <= s->halow[0]; x++) {
				double xd2 = x != 0 ? pow((abs(x) - 1) * s->cellLength[0], 2) : 0;
				if (xd2 + yd2 + zd2 <= rc2) {
					long off = cell_index_3d(s, x, y, z);
					if (off > 0 && s->nfwd < 512) s->fwd[s->nfwd++] = off;
					if (off < 0 && s->nbwd < 512) s->bwd[s->nbwd++] = off;
				}
			}
		}
	}
	s->cells_valid = 0;
	return ORC_OK;
}

orc_sys* orc_create(const double length[3], double rc, double rcLJ, double cells_in_cutoff, int ncomp,
                    const double* eps, const double* sigma, const double* mass, const int* do_shift,
                    const double* mix) {
	orc_sys* s = (orc_sys*) calloc(1, sizeof(orc_sys));
	for (int d = 0; d < 3; d++) s->L[d] = length[d];
	s->rc = rc;
	s->rcLJ = rcLJ == 0.0 ? rc : rcLJ;
	s->cic = cells_in_cutoff;
	s->ncomp = ncomp;
	size_t n2 = (size_t) ncomp * ncomp;
	s->eps24 = (double*) calloc(n2, sizeof(double));
	s->sig2 = (double*) calloc(n2, sizeof(double));
	s->shift6 = (double*) calloc(n2, sizeof(double));
	s->mass = (double*) malloc(ncomp * sizeof(double));
	s->eps = (double*) malloc(ncomp * sizeof(double));
	s->sigma = (double*) malloc(ncomp * sizeof(double));
	s->do_shift = (int*) malloc(ncomp * sizeof(int));
	for (int i = 0; i < ncomp; i++) {
		s->mass[i] = mass[i];
		s->eps[i] = eps[i];
		s->sigma[i] = sigma[i];
		s->do_shift[i] = do_shift[i];
	}
	init_params(s, mix);
	s->order_cap = 1024;
	s->order_buf = (long*) malloc((size_t) s->order_cap * sizeof(long));
	s->head = s->tail = s->order_cap;
	s->beta_trans = 1.0;
	s->T_target = 1.0;
	s->status = init_cells(s);
	return s;
}

void orc_destroy(orc_sys* s) {
	if (!s) return;
	if (s->cells)
		for (long c = 0; c < s->ncells; c++) free(s->cells[c].item);
	free(s->cells);
	free(s->region);
	free(s->inner);
	free(s->boundary);
	free(s->halo);
	free(s->pool);
	free(s->order_buf);
	free(s->eps24);
	free(s->sig2);
	free(s->shift6);
	free(s->mass);
	free(s->eps);
	free(s->sigma);
	free(s->do_shift);
	free(s->rdf_counts);
	free(s);
}

int orc_status(const orc_sys* s) { return s->status; }

/* ---------------------------------------------------------------- container */

/* Whether floor((r - haloMin) / cellLength) names a cell of the halo-inclusive grid. A position
 * inside the halo box can fail this: an image placed by exchangeMolecules within an ulp of the
 * halo box's upper face (a molecule exactly on a cell face, r + L rounding up to haloMax) gives
 * an index one past the last cell. */
static int cell_in_range(const orc_sys* s, const double r[3]) {
	for (int d = 0; d < 3; d++) {
		const int ci = (int) floor((r[d] - s->haloMin[d]) / s->cellLength[d]);
		if (ci < 0 || ci >= s->cpd[d]) return 0;
	}
	return 1;
}

/* LinkedCells::addParticle, LinkedCells.cpp:182-204.
 * One departure from the reference: where its cell index runs one past the cell array (see
 * cell_in_range) the reference writes beyond the array (undefined behaviour: the compiled reference
 * crashes); here that image is not added. It lies a cell length (>= cutoff) beyond every molecule of
 * the box, so it has no partner within the cutoff and the forces, Upot and virial are unchanged. */
static void add_particle(orc_sys* s, const orc_mol* m) {
	if (!in_halo_box(s, m->r)) return;
	if (!cell_in_range(s, m->r)) return;
	long idx = pool_new(s);
	s->pool[idx] = *m;
	list_push_front(s, idx);
	if (s->cells_valid) cell_push(&s->cells[orc_cell_index(s, m->r)], idx);
}

/* InputOldstyle::readPhaseSpace, InputOldstyle.cpp:324-378 (new molecules start with F = 0) */
int orc_add_particles(orc_sys* s, long n, const unsigned long* id, const int* cid, const double* r,
                      const double* v) {
	if (s->status) return s->status;
	for (long i = 0; i < n; i++) {
		if (cid[i] < 0 || cid[i] >= s->ncomp) return s->status = ORC_ERR_ARGS;
		orc_mol m;
		memset(&m, 0, sizeof(m));
		m.id = id[i];
		m.cid = cid[i];
		for (int d = 0; d < 3; d++) {
			m.r[d] = r[3 * i + d];
			m.v[d] = v[3 * i + d];
		}
		add_particle(s, &m);
	}
	return ORC_OK;
}

/* LinkedCells::update, LinkedCells.cpp:165-180 */
int orc_update(orc_sys* s) {
	if (s->status) return s->status;
	for (long c = 0; c < s->ncells; c++) s->cells[c].n = 0;
	for (long k = s->head; k < s->tail; k++) {
		long idx = s->order_buf[k];
		if (!in_halo_box(s, s->pool[idx].r)) return s->status = ORC_ERR_OUTSIDE_HALO;
		cell_push(&s->cells[orc_cell_index(s, s->pool[idx].r)], idx);
	}
	s->cells_valid = 1;
	return ORC_OK;
}

/* LinkedCells::deleteOuterParticles, LinkedCells.cpp:339-371. The pool is compacted in list order. */
int orc_delete_outer(orc_sys* s) {
	if (s->status) return s->status;
	for (long h = 0; h < s->nhalo; h++) s->cells[s->halo[h]].n = 0;
	long n = 0;
	orc_mol* np = (orc_mol*) malloc((size_t) (s->tail - s->head + 1) * sizeof(orc_mol));
	long* remap = (long*) malloc((size_t) (s->pool_n + 1) * sizeof(long));
	for (long k = 0; k < s->pool_n; k++) remap[k] = -1;
	for (long k = s->head; k < s->tail; k++) {
		const orc_mol* m = &s->pool[s->order_buf[k]];
		int erase = 0;
		for (int d = 0; d < 3; ++d)
			if (m->r[d] < 0.0 || m->r[d] >= s->L[d]) erase = 1;
		if (!erase) {
			remap[s->order_buf[k]] = n;
			np[n++] = *m;
		}
	}
	/* the remaining cells keep pointing at the surviving molecules (std::list nodes do not move) */
	for (long c = 0; c < s->ncells; c++) {
		orc_cell* cl = &s->cells[c];
		long w = 0;
		for (long e = 0; e < cl->n; e++) {
			long nw = cl->item[e] < s->pool_n ? remap[cl->item[e]] : -1;
			if (nw >= 0) cl->item[w++] = nw;
		}
		cl->n = w;
	}
	free(remap);
	free(s->pool);
	s->pool = np;
	s->pool_n = n;
	s->pool_cap = s->tail - s->head + 1;
	if (s->order_cap < 2 * n + 1024) {
		free(s->order_buf);
		s->order_cap = 2 * n + 1024;
		s->order_buf = (long*) malloc((size_t) s->order_cap * sizeof(long));
	}
	s->head = s->order_cap - n;
	s->tail = s->order_cap;
	for (long i = 0; i < n; i++) s->order_buf[s->head + i] = i;
	return ORC_OK;
}

/* DomainDecompDummy::exchangeMolecules, DomainDecompDummy.cpp:22-116 (sequential halo images).
 * Images are new molecules with the source's id, component and velocity, F = 0. */
int orc_exchange(orc_sys* s) {
	if (s->status) return s->status;
	for (int d = 0; d < 3; ++d) {
		double psize = s->L[d] - 0.0;
		double low = 0.0 + s->haloLength[d];
		double high = s->L[d] - s->haloLength[d];
		/* images go to the front; the molecules present at begin() stay the last `count` entries
		 * of the list even when the order buffer is reallocated */
		long count = s->tail - s->head;
		for (long i = 0; i < count; i++) {
			orc_mol src = s->pool[s->order_buf[s->tail - count + i]];
			double rd = src.r[d];
			if (rd < low || rd >= high) {
				orc_mol m;
				memset(&m, 0, sizeof(m));
				m.id = src.id;
				m.cid = src.cid;
				for (int d2 = 0; d2 < 3; d2++) {
					m.r[d2] = src.r[d2];
					m.v[d2] = src.v[d2];
				}
				m.r[d] = rd < low ? rd + psize : rd - psize;
				add_particle(s, &m);
			}
		}
	}
	return ORC_OK;
}

/* Compensated (double-double) accumulation, used only for the exactly-summed energy and virial
 * the tests compare against; the reference's own sums are kept separately. */
static void dd_add(double* hi, double* lo, double x) {
	double s = *hi + x;
	double bp = s - *hi;
	double err = (*hi - (s - bp)) + (x - bp);
	*hi = s;
	*lo += err;
}

/* Molecule::isLessThan, Molecule.cpp:439-461 */
static int is_less_than(const orc_mol* a, const orc_mol* b, int* err) {
	if (a->r[2] < b->r[2]) return 1;
	if (a->r[2] > b->r[2]) return 0;
	if (a->r[1] < b->r[1]) return 1;
	if (a->r[1] > b->r[1]) return 0;
	if (a->r[0] < b->r[0]) return 1;
	if (a->r[0] > b->r[0]) return 0;
	*err = 1;
	return 0;
}

/* ParticlePairs2PotForceAdapter::processPair (ParticlePairs2PotForceAdapter.h:84-115) for one
 * LJ centre per molecule: PotForce LJ loop (potforce.h:328-363) and PotForceLJ (potforce.h:41-53).
 * drm = r1 - r2 (Molecule::dist2, Molecule.h:135-142 called as m2.dist2(m1)). */
static void process_pair(orc_sys* s, orc_mol* m1, orc_mol* m2, const double drm[3], int mol_mol, double dd,
                         int calculateLJ, double* upot6, double* virial) {
	s->npairs += 1.0;
	if (mol_mol && s->rdf_on) {
		/* RDF::observeRDF, RDF.h:76-82 */
		if (!(dd > s->rdf_max2)) {
			unsigned l = (unsigned) floor(sqrt(dd) / s->rdf_interval);
			if ((int) l < s->rdf_bins) s->rdf_counts[l]++;
		}
	}
	int n = s->ncomp;
	double eps24 = s->eps24[m1->cid * n + m2->cid];
	double sig2 = s->sig2[m1->cid * n + m2->cid];
	double shift6 = s->shift6[m1->cid * n + m2->cid];
	double drs[3], dr2;
	/* SiteSiteDistance with both sites at the molecule centre, potforce.h:26-31 */
	for (int d = 0; d < 3; ++d) drs[d] = drm[d] + 0.0 - 0.0;
	dr2 = drs[0] * drs[0] + drs[1] * drs[1] + drs[2] * drs[2];
	if (!calculateLJ) return;
	double invdr2 = 1. / dr2;
	double lj6 = sig2 * invdr2;
	lj6 = lj6 * lj6 * lj6;
	double lj12 = lj6 * lj6;
	double lj12m6 = lj12 - lj6;
	double u = eps24 * lj12m6;
	double fac = eps24 * (lj12 + lj12m6) * invdr2;
	double f[3];
	for (int d = 0; d < 3; ++d) f[d] = fac * drs[d];
	u += shift6;
	for (int d = 0; d < 3; ++d) m1->F[d] += f[d];
	for (int d = 0; d < 3; ++d) m2->F[d] -= f[d];
	*upot6 += u;
	for (int d = 0; d < 3; ++d) *virial += drm[d] * f[d];
	if (mol_mol) {
		dd_add(&s->u6_hi, &s->u6_lo, u);
		dd_add(&s->w_hi, &s->w_lo, drm[0] * f[0] + drm[1] * f[1] + drm[2] * f[2]);
	}
}

/* BlockTraverse::traversePairs, BlockTraverse.cpp:89-350 (LJ part; Tersoff passes are no-ops for
 * LJ molecules), with ParticlePairs2PotForceAdapter::init/finish (.h:52-67).  Molecule F doubles
 * as the LJ-centre force: it is zeroed here (BlockTraverse.cpp:110-121; upd_cache/clearFM also
 * zero the site forces) and Molecule::calcFM's F += F_site adds to an exact zero. */
int orc_traverse(orc_sys* s) {
	if (s->status) return s->status;
	if (!s->cells_valid) return s->status = ORC_ERR_ARGS;
	double upot6 = 0, virial = 0, dummy6, dummyv;
	double rc2 = s->rc * s->rc, rcLJ2 = s->rcLJ * s->rcLJ;
	int err = 0;
	s->npairs = 0;
	s->u6_hi = s->u6_lo = s->w_hi = s->w_lo = 0.0;
	for (long k = s->head; k < s->tail; k++) {
		orc_mol* m = &s->pool[s->order_buf[k]];
		m->F[0] = m->F[1] = m->F[2] = 0.0;
	}
	double dr[3];
#define ORC_DIST2(m1, m2, dd)                        \
	do {                                             \
		dd = 0.;                                     \
		for (int d_ = 0; d_ < 3; d_++) {             \
			dr[d_] = (m1)->r[d_] - (m2)->r[d_];      \
			dd += dr[d_] * dr[d_];                   \
		}                                            \
	} while (0)
	/* inner cells: self + forward neighbours, BlockTraverse.cpp:136-189 */
	for (long ii = 0; ii < s->ninner; ii++) {
		long ci = s->inner[ii];
		orc_cell* c = &s->cells[ci];
		if (c->n == 0) continue;
		for (long a = 0; a < c->n; a++) {
			orc_mol* m1 = &s->pool[c->item[a]];
			for (long b = a + 1; b < c->n; b++) {
				orc_mol* m2 = &s->pool[c->item[b]];
				double dd;
				ORC_DIST2(m1, m2, dd);
				if (dd < rc2) process_pair(s, m1, m2, dr, 1, dd, dd < rcLJ2, &upot6, &virial);
			}
		}
		for (int f = 0; f < s->nfwd; f++) {
			orc_cell* nc = &s->cells[ci + s->fwd[f]];
			if (nc->n == 0) continue;
			for (long a = 0; a < c->n; a++) {
				orc_mol* m1 = &s->pool[c->item[a]];
				for (long b = 0; b < nc->n; b++) {
					orc_mol* m2 = &s->pool[nc->item[b]];
					double dd;
					ORC_DIST2(m1, m2, dd);
					if (dd < rc2) process_pair(s, m1, m2, dr, 1, dd, dd < rcLJ2, &upot6, &virial);
				}
			}
		}
	}
	/* boundary cells: self, forward (halo pairs typed by isLessThan), backward halo only,
	 * BlockTraverse.cpp:236-320 */
	for (long bi = 0; bi < s->nboundary; bi++) {
		long ci = s->boundary[bi];
		orc_cell* c = &s->cells[ci];
		if (c->n == 0) continue;
		for (long a = 0; a < c->n; a++) {
			orc_mol* m1 = &s->pool[c->item[a]];
			for (long b = a + 1; b < c->n; b++) {
				orc_mol* m2 = &s->pool[c->item[b]];
				double dd;
				ORC_DIST2(m1, m2, dd);
				if (dd < rc2) process_pair(s, m1, m2, dr, 1, dd, dd < rcLJ2, &upot6, &virial);
			}
		}
		for (int f = 0; f < s->nfwd; f++) {
			long nci = ci + s->fwd[f];
			orc_cell* nc = &s->cells[nci];
			if (nc->n == 0) continue;
			for (long a = 0; a < c->n; a++) {
				orc_mol* m1 = &s->pool[c->item[a]];
				for (long b = 0; b < nc->n; b++) {
					orc_mol* m2 = &s->pool[nc->item[b]];
					double dd;
					ORC_DIST2(m1, m2, dd);
					if (dd < rc2) {
						int mm = 1;
						if (s->region[nci] == 0 && !is_less_than(m1, m2, &err)) mm = 0;
						if (mm)
							process_pair(s, m1, m2, dr, 1, dd, dd < rcLJ2, &upot6, &virial);
						else {
							dummy6 = 0.0;
							process_pair(s, m1, m2, dr, 0, dd, dd < rcLJ2, &dummy6, &dummyv);
						}
					}
				}
			}
		}
		for (int f = 0; f < s->nbwd; f++) {
			long nci = ci + s->bwd[f];
			orc_cell* nc = &s->cells[nci];
			if (s->region[nci] == 0 && nc->n > 0) {
				for (long a = 0; a < c->n; a++) {
					orc_mol* m1 = &s->pool[c->item[a]];
					for (long b = 0; b < nc->n; b++) {
						orc_mol* m2 = &s->pool[nc->item[b]];
						double dd;
						ORC_DIST2(m1, m2, dd);
						if (dd < rc2) {
							int mm = is_less_than(m1, m2, &err);
							if (mm)
								process_pair(s, m1, m2, dr, 1, dd, dd < rcLJ2, &upot6, &virial);
							else {
								dummy6 = 0.0;
								process_pair(s, m1, m2, dr, 0, dd, dd < rcLJ2, &dummy6, &dummyv);
							}
						}
					}
				}
			}
		}
	}
#undef ORC_DIST2
	if (err) return s->status = ORC_ERR_SAME_POSITION;
	/* ParticlePairs2PotForceAdapter::finish, .h:64-67 (no polarity, Tersoff or RF terms) */
	s->local_upot = upot6 / 6. + 0.0 + 0.0 + 0.0;
	s->local_virial = virial + 3.0 * 0.0;
	return ORC_OK;
}

/* ---------------------------------------------------------------- integrator and domain */

/* Domain::initFarFieldCorr, Domain.cpp:574-677, for single LJ centres at the molecule origin
 * (tau1 = tau2 = 0 => TICCu/TICCv, CutoffCorrections.cpp:10-32) and no polar sites. */
static double ticc_u(int n, double rc, double sigma2) { return -pow(rc, 2 * n + 3) / (pow(sigma2, n) * (2 * n + 3)); }
static double ticc_v(int n, double rc, double sigma2) { return 2 * n * ticc_u(n, rc, sigma2); }

static void far_field_corr(orc_sys* s, const long* ncomp_count, long nmol, double rho) {
	double UpotCorrLJ = 0., VirialCorrLJ = 0.;
	int n = s->ncomp;
	for (int i = 0; i < n; ++i)
		for (int j = 0; j < n; ++j) {
			double eps24 = s->eps24[i * n + j], sig2 = s->sig2[i * n + j], sh = s->shift6[i * n + j];
			if (sh == 0.0) {
				double fac = (double) ncomp_count[i] * (double) ncomp_count[j] * eps24;
				UpotCorrLJ += fac * (ticc_u(-6, s->rcLJ, sig2) - ticc_u(-3, s->rcLJ, sig2));
				VirialCorrLJ += fac * (ticc_v(-6, s->rcLJ, sig2) - ticc_v(-3, s->rcLJ, sig2));
			}
		}
	double fac = M_PI * rho / (3. * nmol);
	UpotCorrLJ *= fac;
	VirialCorrLJ *= -fac;
	s->upot_corr = UpotCorrLJ + 0.0;
	s->virial_corr = VirialCorrLJ + 3. * 0.0;
}

/* Domain::calculateGlobalValues, Domain.cpp:158-263 (one thermostat, no rotational DOF). */
static int global_values(orc_sys* s, double tfactor) {
	s->global_upot = s->local_upot + s->upot_corr;
	s->global_virial = s->local_virial + s->virial_corr;
	unsigned long nmol = (unsigned long) (s->tail - s->head);
	double summv2 = s->summv2, sumIw2 = 0.0;
	unsigned long rotDOF = 0;
	s->T = nmol > 0 ? (summv2 + sumIw2) / (double) (3 * nmol + rotDOF) : s->T_target;
	double Ti = tfactor * s->T_target;
	if (Ti > 0.0 && !s->nve)
		s->beta_trans = pow(3.0 * nmol * Ti / summv2, 0.4);
	else
		s->beta_trans = 1.0;
	if (s->beta_trans < 0.9) return s->status = ORC_ERR_EXPLOSION; /* MIN_BETA, Domain.h:33 */
	return ORC_OK;
}

static double summv2_of(orc_sys* s) {
	/* sum m v^2 accumulated in container order (Leapfrog.cpp:75-81, Molecule.cpp:198-205) */
	double sum = 0.0;
	for (long k = s->head; k < s->tail; k++) {
		const orc_mol* m = &s->pool[s->order_buf[k]];
		double v2 = 0.;
		for (int d = 0; d < 3; ++d) v2 += m->v[d] * m->v[d];
		sum += s->mass[m->cid] * v2;
	}
	return sum;
}

/* Simulation::initConfigOldstyle tail, Simulation.cpp:866-877, plus InputOldstyle's global rho
 * (InputOldstyle.cpp:384-387) and the NVE token (Simulation.cpp:851-852). */
int orc_init(orc_sys* s, double target_temperature, int nve) {
	if (s->status) return s->status;
	s->T_target = target_temperature;
	s->nve = nve;
	long nmol = s->tail - s->head;
	long* cnt = (long*) calloc((size_t) s->ncomp, sizeof(long));
	for (long k = s->head; k < s->tail; k++) cnt[s->pool[s->order_buf[k]].cid]++;
	double rho = nmol / (s->L[0] * s->L[1] * s->L[2]);
	far_field_corr(s, cnt, nmol, rho);
	free(cnt);
	int st = orc_update(s);
	if (st) return st;
	return orc_delete_outer(s);
}

/* Simulation::prepare_start, Simulation.cpp:907-947 */
int orc_prepare_start(orc_sys* s) {
	int st;
	if ((st = orc_delete_outer(s))) return st;
	if ((st = orc_update(s))) return st;
	if ((st = orc_exchange(s))) return st;
	if ((st = orc_traverse(s))) return st;
	if ((st = orc_delete_outer(s))) return st;
	s->summv2 = summv2_of(s);
	s->summv2_end = s->summv2;
	return global_values(s, 1.0);
}

/* Simulation::simulateStep, Simulation.cpp:1218-1229, for an NVE or single-thermostat LJ run:
 * Leapfrog::transition1to2 (Leapfrog.cpp:37-51) with Molecule::upd_preF (Molecule.cpp:128-135),
 * update + exchange, traversePairs, deleteOuterParticles, Leapfrog::transition2to3
 * (Leapfrog.cpp:53-99) with Molecule::upd_postF (Molecule.cpp:193-205), calculateGlobalValues and
 * the velocity scaling of Simulation::thermostatEtc (Simulation.cpp:1155-1179). */
int orc_step(orc_sys* s, double dt, double tfactor) {
	int st;
	if (s->status) return s->status;
	double vcorr = 2. - 1. / s->beta_trans;
	for (long k = s->head; k < s->tail; k++) {
		orc_mol* m = &s->pool[s->order_buf[k]];
		double dt_halve = .5 * dt;
		double dtInv2m = dt_halve / s->mass[m->cid];
		for (int d = 0; d < 3; ++d) {
			m->v[d] = vcorr * m->v[d] + dtInv2m * m->F[d];
			m->r[d] += dt * m->v[d];
		}
	}
	if ((st = orc_update(s))) return st;
	if ((st = orc_exchange(s))) return st;
	if ((st = orc_traverse(s))) return st;
	if ((st = orc_delete_outer(s))) return st;
	double dt_half = 0.5 * dt;
	double summv2 = 0.0;
	for (long k = s->head; k < s->tail; k++) {
		orc_mol* m = &s->pool[s->order_buf[k]];
		double dtInv2m = dt_half / s->mass[m->cid];
		double v2 = 0.;
		for (int d = 0; d < 3; ++d) {
			m->v[d] += dtInv2m * m->F[d];
			v2 += m->v[d] * m->v[d];
		}
		summv2 += s->mass[m->cid] * v2;
	}
	s->summv2 = summv2;
	if ((st = global_values(s, tfactor))) return st;
	if (!s->nve) {
		for (long k = s->head; k < s->tail; k++) {
			orc_mol* m = &s->pool[s->order_buf[k]];
			for (int d = 0; d < 3; ++d) m->v[d] *= s->beta_trans;
		}
	}
	s->summv2_end = summv2_of(s);
	return ORC_OK;
}

/* ---------------------------------------------------------------- queries */

long orc_count(const orc_sys* s) { return s->tail - s->head; }

void orc_get(const orc_sys* s, unsigned long* id, int* cid, double* r, double* v, double* F, long* cell) {
	long i = 0;
	for (long k = s->head; k < s->tail; k++, i++) {
		const orc_mol* m = &s->pool[s->order_buf[k]];
		if (id) id[i] = m->id;
		if (cid) cid[i] = m->cid;
		for (int d = 0; d < 3; d++) {
			if (r) r[3 * i + d] = m->r[d];
			if (v) v[3 * i + d] = m->v[d];
			if (F) F[3 * i + d] = m->F[d];
		}
		if (cell) cell[i] = orc_cell_index(s, m->r);
	}
}

void orc_scalars(const orc_sys* s, double* out) {
	out[0] = s->local_upot;
	out[1] = s->local_virial;
	out[2] = s->summv2;
	out[3] = s->global_upot;
	out[4] = s->global_virial;
	out[5] = s->T;
	out[6] = s->beta_trans;
	out[7] = s->upot_corr;
	out[8] = s->virial_corr;
	out[9] = s->npairs;
	out[10] = s->summv2_end;
	out[11] = (s->u6_hi + s->u6_lo) / 6.;
	out[12] = s->w_hi + s->w_lo;
}

void orc_geometry(const orc_sys* s, int* oi, double* od) {
	for (int d = 0; d < 3; d++) {
		oi[d] = s->boxw[d];
		oi[3 + d] = s->halow[d];
		oi[6 + d] = s->cpd[d];
		od[d] = s->cellLength[d];
		od[3 + d] = s->haloMin[d];
		od[6 + d] = s->haloMax[d];
	}
}

void orc_params(const orc_sys* s, int ci, int cj, double* out3) {
	int n = s->ncomp;
	out3[0] = s->eps24[ci * n + cj];
	out3[1] = s->sig2[ci * n + cj];
	out3[2] = s->shift6[ci * n + cj];
}

void orc_rdf_enable(orc_sys* s, double interval, int bins) {
	free(s->rdf_counts);
	s->rdf_counts = (unsigned long*) calloc((size_t) bins, sizeof(unsigned long));
	s->rdf_on = bins > 0;
	s->rdf_bins = bins;
	s->rdf_interval = interval;
	s->rdf_max2 = interval * interval * bins * bins; /* RDF.cpp:30 */
}

void orc_rdf_counts(const orc_sys* s, unsigned long* out) {
	for (int i = 0; i < s->rdf_bins; i++) out[i] = s->rdf_counts[i];
}
