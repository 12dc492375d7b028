/*
 * dg_cuda.c -- the reference-side binding of the B200 path (see dg_cuda.h).
 *
 * C99, compiled with the reference's own sources and headers; the only
 * interface to the GPU is include/gdon3d_cuda.h.  A side table keyed by the
 * gdn_simulation pointer holds the attach handles, so the reference's
 * structs keep their layout.
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <dg/dg.h>
#include <mesh/mesh.h>
#include <mesh/t10.h>
#include <models/d3q4.h>
#include <models/d3q6.h>
#include <models/maxwell.h>
#include <models/model.h>
#include <simulation/simulation.h>

#include "dg_cuda.h"

#define DG_CUDA_MAX_ATTACHED 64
/* volume-node sample of the descriptor check: at most this many elements */
#define DG_CUDA_CHECK_ELEMS 65536
/* theta of the reference's Crank-Nicolson transport (src/dg/relaxation.c:133) */
#define DG_CUDA_THETA 0.5

typedef struct dg_cuda_entry {
	gdn_simulation *simu;
	gdn_cuda_handle *h;
	const gdn_mesh *mesh; /* what the handle was built from */
	double dt;
	int kinetic;
	int routed; /* attached by dg_cuda_route_all */
	int status; /* of the last routed dg_solve */
	double attach_s; /* wall time of the attach, reported as cpu_assembly_t */
} dg_cuda_entry;

static dg_cuda_entry g_tab[DG_CUDA_MAX_ATTACHED];
static int g_route;
static gdn_cuda_data g_route_data;
static gdn_cuda_config g_route_cfg;
static char g_msg[512];
static double g_mismatch;

static int fail(int code, const char *fmt, ...)
{
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
	va_end(ap);
	return code;
}

const char *dg_cuda_message(void)
{
	return g_msg;
}

double dg_cuda_data_mismatch(void)
{
	return g_mismatch;
}

static dg_cuda_entry *find(const gdn_simulation *simu)
{
	for (int i = 0; i < DG_CUDA_MAX_ATTACHED; i++)
		if (g_tab[i].simu == simu && g_tab[i].h)
			return &g_tab[i];
	return NULL;
}

static double wall_s(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* The P2 tables through the reference's accessors (src/mesh/t10.h:72-86). */
static void reference_tables(gdn_cuda_tables *t)
{
	for (int i = 0; i < 10; i++) {
		t->wpg[i] = t10_get_wpg_ref_entry(i);
		for (int j = 0; j < 10; j++) {
			t->mass[i][j] = t10_get_mass_ref_entry(i, j);
			t->inv_mass[i][j] = t10_get_inv_mass_ref_entry(i, j);
			for (int k = 0; k < 3; k++)
				t->internal[i][j][k] = t10_get_internal_ref_entry(i, j, k);
		}
	}
	for (int i = 0; i < 6; i++)
		for (int j = 0; j < 6; j++)
			t->face_scal[i][j] = t10_get_face_scale_entry(i, j);
	for (int f = 0; f < 4; f++) {
		for (int k = 0; k < 3; k++)
			t->ref_normal[f][k] = t10_get_ref_normal_entry(f, k);
		for (int j = 0; j < 6; j++)
			t->face2node[f][j] = t10_get_ref_face2node_entry(f, j);
	}
}

/* gdn_model (src/models/model.h:41-62) -> the physics the device runs. */
static int device_model(const gdn_simulation *simu, gdn_cuda_model *cm)
{
	const gdn_model *mo = simu->mdl;
	memset(cm, 0, sizeof(*cm));
	if (!mo || mo->nb_w != 6 || mo->get_num_flux != maxwell_num_flux_upwind)
		return fail(GDN_CUDA_ERR_UNSUPPORTED, "dg_cuda: only Maxwell with maxwell_num_flux_upwind runs on the GPU");
	if (!mo->get_imposed_data)
		return fail(GDN_CUDA_ERR_INVALID, "dg_cuda: the model has no get_imposed_data");
	cm->nb_w = 6;
	cm->theta = DG_CUDA_THETA;
	if (mo->get_num_flux_boundary == maxwell_num_flux_upwind)
		cm->boundary_flux = GDN_CUDA_BC_UPWIND;
	else if (mo->get_num_flux_boundary == maxwell_num_flux_boundary_metal && !simu->use_kinetic_scheme)
		cm->boundary_flux = GDN_CUDA_BC_METAL;
	else
		return fail(GDN_CUDA_ERR_UNSUPPORTED, "dg_cuda: unsupported boundary flux for this scheme");
	if (!simu->use_kinetic_scheme) {
		cm->scheme = GDN_CUDA_SCHEME_RK3;
		cm->lambda = mo->lambda;
		return GDN_CUDA_OK;
	}
	/* the kinetic scheme: the velocity set is recognised by its functions */
	const int d3q4 = mo->get_feq == d3q4_get_feq && mo->get_w == d3q4_get_w && mo->get_fR == d3q4_get_fR;
	const int d3q6 = mo->get_feq == d3q6_get_feq && mo->get_w == d3q6_get_w && mo->get_fR == d3q6_get_fR;
	if (!(d3q4 && mo->nb_v == 4) && !(d3q6 && mo->nb_v == 6))
		return fail(GDN_CUDA_ERR_UNSUPPORTED, "dg_cuda: kinetic velocity sets d3q4 and d3q6 only");
	cm->scheme = GDN_CUDA_SCHEME_KINETIC;
	cm->nb_v = mo->nb_v;
	cm->lambda = mo->lambda;
	cm->omega = mo->omega;
	cm->vi = mo->vi;
	return GDN_CUDA_OK;
}

/* The descriptor against model->get_imposed_data: every boundary node
 * (dg_update_boundary's points, src/dg/dg.c:84-93) at t = 0 and t = dt, the
 * volume nodes of evenly spaced elements at t = 0 (dg_init_sol_macro's
 * points, dg.c:42-58).  Evaluated on the device by the solver's own code. */
static int check_descriptor(const gdn_simulation *simu, const gdn_cuda_data *data, int device)
{
	const gdn_mesh *mesh = simu->tt;
	const long long nbf = mesh->nboundaryfaces, ne = mesh->nbelems;
	const long long stride = ne > DG_CUDA_CHECK_ELEMS ? (ne + DG_CUDA_CHECK_ELEMS - 1) / DG_CUDA_CHECK_ELEMS : 1;
	const long long nvol = (ne + stride - 1) / stride * 10;
	const long long nb = nbf * 6;
	const long long npts = nb > nvol ? nb : nvol;
	double *xyz = malloc(sizeof(double) * 3 * (npts > 0 ? npts : 1));
	double *wd = malloc(sizeof(double) * 6 * (npts > 0 ? npts : 1));
	if (!xyz || !wd) {
		free(xyz);
		free(wd);
		return fail(GDN_CUDA_ERR_OOM, "dg_cuda: host allocation failed");
	}
	double worst = 0.0, wmax = 0.0;
	int rc = GDN_CUDA_OK;
	for (int pass = 0; pass < 3 && rc == GDN_CUDA_OK; pass++) {
		const double t = pass == 1 ? simu->dt : 0.0;
		long long n = 0;
		if (pass < 2) {
			for (long long f = 0; f < nbf; f++)
				for (int j = 0; j < 6; j++) {
					const int ipg = mesh_get_ipg_elem_left_from_face(mesh, mesh->boundaryface[f], j);
					memcpy(xyz + 3 * n++, mesh->node + 3 * mesh->elem2qnode[ipg], 3 * sizeof(double));
				}
		} else {
			for (long long e = 0; e < ne; e += stride)
				for (int i = 0; i < 10; i++)
					memcpy(xyz + 3 * n++, mesh->node + 3 * mesh->elem2qnode[10 * e + i], 3 * sizeof(double));
		}
		rc = gdn_cuda_eval_data(data, n, xyz, t, wd, device);
		if (rc != GDN_CUDA_OK) {
			fail(rc, "dg_cuda: %s", gdn_cuda_last_error());
			break;
		}
		for (long long i = 0; i < n; i++) {
			double wc[6];
			simu->mdl->get_imposed_data(xyz + 3 * i, t, wc);
			for (int c = 0; c < 6; c++) {
				const double d = fabs(wc[c] - wd[6 * i + c]);
				if (!(d <= worst)) /* NaN counts as a mismatch */
					worst = d;
				if (fabs(wc[c]) > wmax)
					wmax = fabs(wc[c]);
			}
		}
	}
	free(xyz);
	free(wd);
	if (rc != GDN_CUDA_OK)
		return rc;
	g_mismatch = worst / (wmax > 1.0 ? wmax : 1.0);
	if (!(g_mismatch <= DG_CUDA_DATA_TOL))
		return fail(GDN_CUDA_ERR_INVALID,
					"dg_cuda: the analytic-data descriptor differs from get_imposed_data by %.3e "
					"(relative to max(1, |w|)), above the %.0e tolerance",
					g_mismatch, DG_CUDA_DATA_TOL);
	return GDN_CUDA_OK;
}

static gdn_cuda_config default_config(void)
{
	gdn_cuda_config c;
	c.precision = GDN_CUDA_FP64;
	c.refine_passes = 1;
	c.rk3_variant = 0;
	c.use_graph = 1;
	c.device = 0;
	c.kin_sweep = 0;
	return c;
}

static void release(dg_cuda_entry *e)
{
	if (e->h)
		gdn_cuda_detach(e->h);
	memset(e, 0, sizeof(*e));
}

static int attach_entry(gdn_simulation *simu, const gdn_cuda_data *data, const gdn_cuda_config *cfg, int routed)
{
	if (!simu || !simu->tt || !simu->mdl || !data)
		return fail(GDN_CUDA_ERR_INVALID, "dg_cuda_attach: simulation, mesh, model and data are needed");
	if (!(simu->dt > 0.0))
		return fail(GDN_CUDA_ERR_INVALID, "dg_cuda_attach: call simulation_set_time_parameters first (dt <= 0)");
	const gdn_cuda_config c = cfg ? *cfg : default_config();
	gdn_cuda_model cm;
	int rc = device_model(simu, &cm);
	if (rc != GDN_CUDA_OK)
		return rc;
	rc = check_descriptor(simu, data, c.device);
	if (rc != GDN_CUDA_OK)
		return rc;
	const gdn_mesh *m = simu->tt;
	gdn_cuda_mesh cmesh = {m->nbelems, m->nbfaces, m->nboundaryfaces, m->nbqnodes_in, m->face2elem,
						   m->fnode2enode, m->boundaryface, m->elem2qnode, m->node};
	gdn_cuda_tables tabs;
	reference_tables(&tabs);
	const double t0 = wall_s();
	gdn_cuda_handle *h = NULL;
	rc = gdn_cuda_attach(&cmesh, &tabs, &cm, data, &c, simu->dt, &h);
	if (rc != GDN_CUDA_OK)
		return fail(rc, "dg_cuda_attach: %s", gdn_cuda_last_error());
	dg_cuda_entry *e = find(simu);
	if (e)
		release(e);
	for (int i = 0; i < DG_CUDA_MAX_ATTACHED && !e; i++)
		if (!g_tab[i].h)
			e = &g_tab[i];
	if (!e) {
		gdn_cuda_detach(h);
		return fail(GDN_CUDA_ERR_INVALID, "dg_cuda_attach: more than %d attached simulations",
					DG_CUDA_MAX_ATTACHED);
	}
	e->simu = simu;
	e->h = h;
	e->mesh = simu->tt;
	e->dt = simu->dt;
	e->kinetic = simu->use_kinetic_scheme;
	e->routed = routed;
	e->status = GDN_CUDA_OK;
	e->attach_s = wall_s() - t0;
	return GDN_CUDA_OK;
}

int dg_cuda_attach(gdn_simulation *simu, const gdn_cuda_data *data, const gdn_cuda_config *cfg)
{
	return attach_entry(simu, data, cfg, 0);
}

int dg_cuda_detach(gdn_simulation *simu)
{
	dg_cuda_entry *e = find(simu);
	if (e)
		release(e);
	return GDN_CUDA_OK;
}

int dg_cuda_route_all(const gdn_cuda_data *data, const gdn_cuda_config *cfg)
{
	if (!data) {
		g_route = 0;
		for (int i = 0; i < DG_CUDA_MAX_ATTACHED; i++)
			if (g_tab[i].h && g_tab[i].routed)
				release(&g_tab[i]);
		return GDN_CUDA_OK;
	}
	g_route_data = *data;
	g_route_cfg = cfg ? *cfg : default_config();
	g_route = 1;
	return GDN_CUDA_OK;
}

int dg_cuda_status(const gdn_simulation *simu)
{
	const dg_cuda_entry *e = find(simu);
	return e ? e->status : GDN_CUDA_OK;
}

int dg_cuda_attached(const gdn_simulation *simu)
{
	return find(simu) != NULL;
}

int dg_cuda_save_all(gdn_simulation *simu, const char *filename, int iternb)
{
	dg_cuda_entry *e = find(simu);
	if (!e)
		return fail(GDN_CUDA_ERR_INVALID, "dg_cuda_save_all: the simulation is not attached");
	const int rc = gdn_cuda_save_xdmf(e->h, 0, filename, iternb);
	if (rc != GDN_CUDA_OK)
		return fail(rc, "dg_cuda_save_all: %s", gdn_cuda_last_error());
	return GDN_CUDA_OK;
}

/* The reference's entry point (src/dg/dg.c:23-30), routed. */
void dg_solve(gdn_simulation *simu)
{
	dg_cuda_entry *e = find(simu);
	/* a routed simulation whose mesh, scheme or dt changed is attached again */
	if (e && e->routed &&
		(e->mesh != simu->tt || e->dt != simu->dt || e->kinetic != (int)simu->use_kinetic_scheme)) {
		release(e);
		e = NULL;
	}
	if (!e && g_route) {
		const int rc = attach_entry(simu, &g_route_data, &g_route_cfg, 1);
		if (rc != GDN_CUDA_OK) {
			fprintf(stderr, "gdon3d_cuda: %s\n", g_msg);
			return; /* no silent CPU fallback */
		}
		e = find(simu);
	}
	if (!e) {
		dg_solve_host(simu);
		return;
	}
	if (e->dt != simu->dt || e->mesh != simu->tt) {
		e->status = fail(GDN_CUDA_ERR_INVALID,
						 "dg_solve: dt or mesh changed since dg_cuda_attach; attach the simulation again");
		fprintf(stderr, "gdon3d_cuda: %s\n", g_msg);
		return;
	}
	e->status = gdn_cuda_solve(e->h, simu->itermax, simu->wn, &simu->t, &simu->cpu_running_t);
	simu->cpu_assembly_t = e->attach_s;
	if (e->status != GDN_CUDA_OK) {
		fail(e->status, "dg_solve: %s", gdn_cuda_last_error());
		fprintf(stderr, "gdon3d_cuda: %s\n", g_msg);
	}
}
