/*
 * ORACLE TEST INFRASTRUCTURE -- not part of the product.
 *
 * Repo-owned driver around the reference's own C code, compiled in place from
 * the reference tree by oracle/Makefile into oracle/_ref/libgdon3d_ref_*.so.
 * It replaces the reference's example programs (examples/*.c) and
 * utils_l2_time_convergence (src/utils/convergence.c:43-98): it builds a mesh
 * with the reference's own reader / connectivity builder, sets up the model
 * exactly like the examples do (examples/rk3_maxwell_plane_wave.c:61-66,
 * examples/relax_maxwell_plane_wave.c:58-65), calls the reference's
 * dg_solve (src/dg/dg.c:23) and simulation_error_l2
 * (src/simulation/simulation.c:606) and hands back the final state vector.
 *
 * The analytic data defined here are the plane wave of the benchmark
 * configurations (a new data set, not in the reference) and the examples'
 * cos wave (imposed_macro_cos, a static function of
 * examples/rk3_maxwell_plane_wave.c:35-47 and
 * examples/relax_maxwell_plane_wave.c:35-47, restated); the PEC cavity and
 * the stationary data use the reference's maxwell_imposed_macro_cavity and
 * maxwell_imposed_stationary (src/models/maxwell.c:118-133, 72-84) directly.
 *
 * Built a third time with GDN_REF_BOUND defined (libgdon3d_ref_bound.so):
 * the reference's dg.c renamed dg_solve -> dg_solve_host and the product's
 * binding integration/dg_cuda.c linked in, so that ref_run_bound drives the
 * reference's own flow with dg_solve routed to the GPU.
 */
#include <math.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <gdon3d.h>
#include <dg/dg.h>
#include <mesh/mesh.h>
#include <mesh/t10.h>
#include <models/d3q4.h>
#include <models/d3q6.h>
#include <models/maxwell.h>
#include <models/model.h>
#include <simulation/simulation.h>

/* analytic data descriptor (same meaning as the product's gdn_cuda_data) */
#include <utils/convergence.h>

#ifdef GDN_REF_BOUND
#include "../integration/dg_cuda.h"
#endif

/* The reference's io_save_all (src/io/io_hdf5.c:355-368) needs libhdf5, which is
 * not installed, so io_hdf5.c is not compiled; utils_l2_time_convergence
 * (src/utils/convergence.c) still names it.  In the bound library an attached
 * simulation is written by the binding (raw binary + XDMF); otherwise nothing
 * is written. */
void io_save_all(gdn_simulation *simulation, char filename[1024], int iternb)
{
#ifdef GDN_REF_BOUND
	if (dg_cuda_attached(simulation)) {
		if (dg_cuda_save_all(simulation, filename, iternb) != 0)
			fprintf(stderr, "io_save_all: %s\n", dg_cuda_message());
		return;
	}
#endif
	(void)simulation;
	(void)iternb;
	fprintf(stderr, "io_save_all: %s not written (no HDF5 writer in this build)\n", filename);
}

typedef struct ref_data {
	int kind; /* 0 plane wave, 1 PEC cavity, 2 stationary (reference formulas),
	             3 the examples' cos wave */
	double khat[3];
	double kmag;
	double pol[3];
	double amp;
	double phase;
} ref_data;

static ref_data g_data;

/* E = amp * pol * sin(kmag (khat.x - t) + phase), H = khat x E */
static void plane_wave(const gdn_real *x, const gdn_real t, gdn_real *w)
{
	const double *k = g_data.khat, *p = g_data.pol;
	double arg = g_data.kmag * ((k[0] * x[0] + k[1] * x[1] + k[2] * x[2]) - t) +
				 g_data.phase;
	double s = g_data.amp * sin(arg);
	double hx = k[1] * p[2] - k[2] * p[1];
	double hy = k[2] * p[0] - k[0] * p[2];
	double hz = k[0] * p[1] - k[1] * p[0];
	w[0] = p[0] * s;
	w[1] = p[1] * s;
	w[2] = p[2] * s;
	w[3] = hx * s;
	w[4] = hy * s;
	w[5] = hz * s;
}

/* the examples' data: Ez = cos(pi (x - t)), Hy = -Ez */
static void example_cos(const gdn_real *x, const gdn_real t, gdn_real *w)
{
	const gdn_real s = cos(1 * M_PI * (x[0] - t));
	w[0] = 0;
	w[1] = 0;
	w[2] = s;
	w[3] = 0;
	w[4] = -s;
	w[5] = 0;
}

static gdn_get_imposed_data select_data(const ref_data *d)
{
	g_data = *d;
	if (d->kind == 1)
		return maxwell_imposed_macro_cavity;
	if (d->kind == 2)
		return maxwell_imposed_stationary;
	if (d->kind == 3)
		return example_cos;
	return plane_wave;
}

void *ref_mesh_from_file(const char *path)
{
	gdn_mesh *m = (gdn_mesh *)calloc(1, sizeof(gdn_mesh));
	mesh_read_from_msh22_file(m, path);
	mesh_build_connectivity(m);
	return m;
}

/* Same state as mesh_read_from_msh22_file leaves (src/mesh/mesh.c:623-726),
 * filled from arrays instead of a file; 0-based elem2node. */
void *ref_mesh_from_arrays(int nbnodes, const double *coords, int nbelems,
						   const int *elem2node)
{
	gdn_mesh *m = (gdn_mesh *)calloc(1, sizeof(gdn_mesh));
	m->nbnodes = nbnodes;
	m->node = (gdn_real *)malloc(sizeof(gdn_real) * 3 * nbnodes);
	memcpy(m->node, coords, sizeof(double) * 3 * nbnodes);
	m->nbelems = nbelems;
	m->elem2node = (int *)malloc(sizeof(int) * 4 * nbelems);
	memcpy(m->elem2node, elem2node, sizeof(int) * 4 * nbelems);
	m->has_physical_groups = false;
	m->is_read = true;
	m->elem2elem = NULL;
	mesh_build_connectivity(m);
	return m;
}

/* The T4 content of a msh22 file as the reference's reader leaves it
 * (src/mesh/mesh.c:623-726, no connectivity): call with NULL arrays for the
 * sizes, then with coords[3*nbnodes] and elem2node[4*nbelems] (0-based). */
int ref_msh_read_raw(const char *path, int *nbnodes, int *nbelems, double *coords, int *elem2node)
{
	gdn_mesh m;
	memset(&m, 0, sizeof(m));
	mesh_read_from_msh22_file(&m, path);
	*nbnodes = m.nbnodes;
	*nbelems = m.nbelems;
	if (coords)
		memcpy(coords, m.node, sizeof(double) * 3 * m.nbnodes);
	if (elem2node)
		memcpy(elem2node, m.elem2node, sizeof(int) * 4 * m.nbelems);
	free(m.node);
	free(m.elem2node);
	if (m.physical_group_is_alloc)
		free(m.physical_group);
	return 0;
}

/* The host callback of data `d` (what model->get_imposed_data returns) at n
 * points and time t: w[6*i + c]. */
void ref_eval_data(const ref_data *d, int n, const double *xyz, double t, double *w)
{
	gdn_get_imposed_data fn = select_data(d);
	for (int i = 0; i < n; i++)
		fn(xyz + 3 * i, t, w + 6 * i);
}

void ref_mesh_info(void *pm, int *out)
{
	gdn_mesh *m = (gdn_mesh *)pm;
	out[0] = m->nbelems;
	out[1] = m->nbfaces;
	out[2] = m->nboundaryfaces;
	out[3] = m->nbqnodes_in;
}

void ref_mesh_arrays(void *pm, int *face2elem, int *fnode2enode,
					 int *boundaryface, int *elem2qnode, double *node)
{
	gdn_mesh *m = (gdn_mesh *)pm;
	memcpy(face2elem, m->face2elem, sizeof(int) * 4 * m->nbfaces);
	memcpy(fnode2enode, m->fnode2enode, sizeof(int) * 12 * m->nbfaces);
	if (m->nboundaryfaces)
		memcpy(boundaryface, m->boundaryface, sizeof(int) * m->nboundaryfaces);
	memcpy(elem2qnode, m->elem2qnode,
		   sizeof(int) * (10 * m->nbelems + 6 * m->nboundaryfaces));
	memcpy(node, m->node, sizeof(double) * 3 * m->nbqnodes_in);
}

double ref_mesh_hmin(void *pm)
{
	return mesh_get_t4_hmin((gdn_mesh *)pm);
}

void ref_mesh_free(void *pm)
{
	gdn_mesh *m = (gdn_mesh *)pm;
	gdn_gdn_mesh_free(m);
	if (m->qnode)
		free(m->qnode);
	free(m);
}

/* scheme: 0 = RK3 Maxwell upwind, 1 = CFL-less d3q4, 2 = CFL-less d3q6,
 * 3 = RK3 Maxwell upwind with the metal boundary flux
 * (maxwell_num_flux_boundary_metal, src/models/maxwell.c:205-223) */
static void setup_model(gdn_model *model, int scheme, const ref_data *d)
{
	memset(model, 0, sizeof(*model));
	model->nb_w = 6;
	model->get_num_flux = maxwell_num_flux_upwind;
	model->get_num_flux_boundary =
		scheme == 3 ? maxwell_num_flux_boundary_metal : maxwell_num_flux_upwind;
	model->get_imposed_data = select_data(d);
	if (scheme == 0 || scheme == 3) {
		model->use_relax_scheme = false;
		model->lambda = 1.0;
	} else {
		model->get_proj_pos = maxwell_get_proj_pos_null_prod_w;
		model->get_proj_neg = maxwell_get_proj_neg_prod_w;
		model->use_relax_scheme = true;
		if (scheme == 1)
			d3q4_set_model(model);
		else
			d3q6_set_model(model);
	}
}

int ref_wlen(void *pm, int scheme)
{
	gdn_mesh *m = (gdn_mesh *)pm;
	int mm = (scheme == 0 || scheme == 3) ? 6 : (scheme == 1 ? 24 : 36);
	return mm * (10 * m->nbelems + 6 * m->nboundaryfaces);
}

/* Runs `steps` time steps of size dt through the reference's dg_solve.
 * tmax is passed as (steps + 0.5) * dt so that simulation_set_time_parameters
 * (src/simulation/simulation.c:144-164) yields itermax == steps.
 * Returns 0, or -1 if the step count did not come out as asked. */
int ref_run(void *pm, int scheme, const ref_data *d, double dt, int steps,
			double *wn_out, double *t_out, double *err_out, double *cpu_run,
			double *cpu_asm)
{
	gdn_mesh *m = (gdn_mesh *)pm;
	gdn_model model;
	gdn_simulation simu;
	memset(&simu, 0, sizeof(simu));
	setup_model(&model, scheme, d);
	simulation_init(m, &model, &simu);
	simulation_set_time_parameters(&simu, (steps + 0.5) * dt, dt, -1);
	if (simu.itermax != steps) {
		free(simu.wn);
		return -1;
	}
	dg_solve(&simu);
	if (wn_out)
		memcpy(wn_out, simu.wn, sizeof(double) * simu.wlen);
	if (t_out)
		*t_out = simu.t;
	if (err_out)
		*err_out = simulation_error_l2(&simu);
	if (cpu_run)
		*cpu_run = simu.cpu_running_t;
	if (cpu_asm)
		*cpu_asm = simu.cpu_assembly_t;
	free(simu.wn);
	return 0;
}

/* L2 error of a given state through the reference's own norm. */
double ref_error_l2(void *pm, int scheme, const ref_data *d, const double *wn,
					double t)
{
	gdn_mesh *m = (gdn_mesh *)pm;
	gdn_model model;
	gdn_simulation simu;
	memset(&simu, 0, sizeof(simu));
	setup_model(&model, scheme, d);
	simulation_init(m, &model, &simu);
	memcpy(simu.wn, wn, sizeof(double) * simu.wlen);
	simu.t = t;
	double e = simulation_error_l2(&simu);
	free(simu.wn);
	return e;
}

/* Initial state through the reference's dg_init_sol_macro (src/dg/dg.c:32). */
void ref_init_state(void *pm, int scheme, const ref_data *d, double *wn_out)
{
	gdn_mesh *m = (gdn_mesh *)pm;
	gdn_model model;
	gdn_simulation simu;
	memset(&simu, 0, sizeof(simu));
	setup_model(&model, scheme, d);
	simulation_init(m, &model, &simu);
	dg_init_sol_macro(&simu);
	memcpy(wn_out, simu.wn, sizeof(double) * simu.wlen);
	free(simu.wn);
}

/* The reference's P2 tables through its public accessors (src/mesh/t10.h:81-86). */
void ref_t10_tables(double *wpg, double *mass, double *inv_mass,
					double *internal, double *face_scal, double *ref_normal,
					int *face2node)
{
	for (int i = 0; i < 10; i++) {
		wpg[i] = t10_get_wpg_ref_entry(i);
		for (int j = 0; j < 10; j++) {
			mass[10 * i + j] = t10_get_mass_ref_entry(i, j);
			inv_mass[10 * i + j] = t10_get_inv_mass_ref_entry(i, j);
			for (int k = 0; k < 3; k++)
				internal[(10 * i + j) * 3 + k] =
					t10_get_internal_ref_entry(i, j, k);
		}
	}
	for (int i = 0; i < 6; i++)
		for (int j = 0; j < 6; j++)
			face_scal[6 * i + j] = t10_get_face_scale_entry(i, j);
	for (int f = 0; f < 4; f++) {
		for (int k = 0; k < 3; k++)
			ref_normal[3 * f + k] = t10_get_ref_normal_entry(f, k);
		for (int j = 0; j < 6; j++)
			face2node[6 * f + j] = t10_get_ref_face2node_entry(f, j);
	}
}

#ifdef GDN_REF_BOUND
/* The reference's flow with the GPU binding: simulation_init,
 * simulation_set_time_parameters, dg_cuda_attach (gd, FP64 or another
 * precision), dg_solve (routed to the GPU), simulation_error_l2 on the state
 * written back.  Returns the attach status (the message through
 * ref_bound_message), or the routed solve's status. */
int ref_run_bound(void *pm, int scheme, const ref_data *d, const gdn_cuda_data *gd, int precision, double dt,
				  int steps, double *wn_out, double *t_out, double *err_out, double *mismatch_out)
{
	gdn_mesh *m = (gdn_mesh *)pm;
	gdn_model model;
	gdn_simulation simu;
	memset(&simu, 0, sizeof(simu));
	setup_model(&model, scheme, d);
	simulation_init(m, &model, &simu);
	simulation_set_time_parameters(&simu, (steps + 0.5) * dt, dt, -1);
	if (simu.itermax != steps) {
		free(simu.wn);
		return -1;
	}
	gdn_cuda_config cfg = {precision, 1, 0, 1, 0, 0};
	int rc = dg_cuda_attach(&simu, gd, &cfg);
	if (mismatch_out)
		*mismatch_out = dg_cuda_data_mismatch();
	if (rc == 0) {
		dg_solve(&simu);
		rc = dg_cuda_status(&simu);
		if (wn_out)
			memcpy(wn_out, simu.wn, sizeof(double) * simu.wlen);
		if (t_out)
			*t_out = simu.t;
		if (err_out)
			*err_out = simulation_error_l2(&simu);
		dg_cuda_detach(&simu);
	}
	free(simu.wn);
	return rc;
}

const char *ref_bound_message(void)
{
	return dg_cuda_message();
}
#endif

/* The reference's own convergence driver utils_l2_time_convergence
 * (src/utils/convergence.c:43-104) on a msh file: nb_run solves from one
 * gdn_simulation with dt halved per run; it prints one line per run (error
 * and order columns, simulation_dump_info, simulation.c:668-692) on stdout.
 * gpu != 0 (bound library only): every dg_solve of the driver is routed to
 * the GPU by dg_cuda_route_all(gd) first.  Returns 0, or the routing status. */
int ref_time_convergence(const char *path, int scheme, const ref_data *d, double init_dt, double tmax,
						 int nb_run, int gpu, const void *gd)
{
	gdn_model model;
	setup_model(&model, scheme, d);
#ifdef GDN_REF_BOUND
	if (gpu && dg_cuda_route_all((const gdn_cuda_data *)gd, NULL) != 0)
		return -1;
#else
	(void)gd;
	if (gpu)
		return -2;
#endif
	utils_l2_time_convergence(&model, nb_run, path, init_dt, tmax, false);
	fflush(stdout);
#ifdef GDN_REF_BOUND
	if (gpu)
		dg_cuda_route_all(NULL, NULL);
#endif
	return 0;
}
