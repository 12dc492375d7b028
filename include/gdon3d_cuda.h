/*
 * gdon3d_cuda.h -- C-ABI of the B200 (sm_100a) implementation of Gdon3d's two
 * data-parallel hot paths:
 *   HP-1  the P2-tetrahedron DG residual driven by the low-storage RK3
 *         (reference: src/dg/explicit.c:39-117, src/simulation/simulation.c
 *          :218-491, src/models/maxwell.c:152-192, src/dg/dg.c:61-107);
 *   HP-2  the CFL-less kinetic-relaxation step: per-velocity Crank-Nicolson
 *         DG transport solves and the relaxation to the Maxwell equilibrium
 *         (reference: src/dg/relaxation.c:24-185, src/simulation/simulation.c
 *          :493-604, src/models/d3q4.c:82-301, src/dg/dg.c:109-147).
 *
 * Plain C types only (ints, doubles, pointers, sizes).  Every call returns an
 * int status (GDN_CUDA_OK = 0) and never aborts; gdn_cuda_last_error() gives
 * the message of the last failure on the calling thread.
 *
 * State vectors passed across this boundary use the reference's layout for
 * gdn_simulation.wn (src/simulation/simulation.h:17-38):
 *   RK3     wn[(ipg) * 6 + iw]            (simulation.c:211-214)
 *   kinetic wn[(iw * nb_v + iv) * neq + ipg]   (simulation.c:22-54)
 * with ipg in [0, neq), neq = 10 * nbelems + 6 * nboundaryfaces: the volume
 * nodes 10 * ie + iloc first, then the boundary dofs 6 * ibf + iloc.
 */
#ifndef GDON3D_CUDA_H
#define GDON3D_CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define GDN_CUDA_OK 0
#define GDN_CUDA_ERR_CUDA 1 /* a CUDA runtime call failed */
#define GDN_CUDA_ERR_INVALID 2 /* bad argument, size or descriptor */
#define GDN_CUDA_ERR_UNSUPPORTED 3 /* model/physics not available on device */
#define GDN_CUDA_ERR_CYCLE 4 /* the upwind element graph has a cycle */
#define GDN_CUDA_ERR_OOM 5 /* device allocation failed */
#define GDN_CUDA_ERR_TIMEOUT 6 /* a bounded device-side wait gave up */
#define GDN_CUDA_ERR_MESH 7 /* inconsistent mesh (bad index, det <= 0) */

/* ---- inputs ------------------------------------------------------------ */

/* The arrays of the reference's gdn_mesh after mesh_build_connectivity
 * (src/mesh/mesh.h:15-45, built at src/mesh/mesh.c:1234-1268). */
typedef struct gdn_cuda_mesh {
	int nbelems;
	int nbfaces;
	int nboundaryfaces;
	int nbqnodes; /* nbqnodes_in */
	const int *face2elem; /* [4*nbfaces] eL, locfaceL, eR (-1), locfaceR (-1) */
	const int *fnode2enode; /* [12*nbfaces] L then R local node ids */
	const int *boundaryface; /* [nboundaryfaces] global face ids */
	const int *elem2qnode; /* [10*nbelems + 6*nboundaryfaces] */
	const double *node; /* [3*nbqnodes] P2 node coordinates */
} gdn_cuda_mesh;

/* The reference's P2 tables, as returned by its accessors
 * t10_get_wpg_ref_entry, t10_get_inv_mass_ref_entry,
 * t10_get_internal_ref_entry, t10_get_face_scale_entry,
 * t10_get_ref_normal_entry, t10_get_ref_face2node_entry
 * (src/mesh/t10.h:72-86).  gdn_cuda_t10_tables() fills the same values. */
typedef struct gdn_cuda_tables {
	double wpg[10];
	double mass[10][10];
	double inv_mass[10][10];
	double internal[10][10][3]; /* [i][j][k] = int d_k(phi_i) phi_j */
	double face_scal[6][6];
	double ref_normal[4][3];
	int face2node[4][6];
} gdn_cuda_tables;

/* Analytic data evaluated on the device (boundary values, initial data and
 * the error norm).  The reference passes a host callback
 * (gdn_model.get_imposed_data, src/models/model.h:24-25); the GPU path needs
 * a descriptor instead.  PLANE: E = amp pol sin(kmag (khat.x - t) + phase),
 * H = khat x E (the examples' cos wave, examples/rk3_maxwell_plane_wave.c
 * :35-47, is khat = (1,0,0), pol = (0,0,1), kmag = pi, phase = pi/2).
 * CAVITY: maxwell_imposed_macro_cavity (src/models/maxwell.c:118-133) with
 * its constants.  STATIONARY: maxwell_imposed_stationary
 * (src/models/maxwell.c:16-84); khat, kmag, pol, amp and phase are unused
 * for CAVITY and STATIONARY.  gdn_cuda_eval_data evaluates a descriptor on
 * the device, so that a host can check it against its callback. */
#define GDN_CUDA_DATA_PLANE 0
#define GDN_CUDA_DATA_CAVITY 1
#define GDN_CUDA_DATA_STATIONARY 2
typedef struct gdn_cuda_data {
	int kind;
	double khat[3];
	double kmag;
	double pol[3];
	double amp;
	double phase;
} gdn_cuda_data;

/* The recognised gdn_model (src/models/model.h:41-62): Maxwell with the
 * upwind flux maxwell_num_flux_upwind (as the boundary flux too, or
 * maxwell_num_flux_boundary_metal for RK3: boundary_flux), either
 * through RK3 (use_relax_scheme = false) or through the CFL-less scheme with
 * the d3q4 (nb_v = 4, d3q4.c:17-42) or d3q6 (nb_v = 6, d3q6.c:18-47)
 * velocity set. */
#define GDN_CUDA_SCHEME_RK3 0
#define GDN_CUDA_SCHEME_KINETIC 1
/* model->get_num_flux_boundary of the RK3 scheme: maxwell_num_flux_upwind
 * with the analytic data as the outside state, or
 * maxwell_num_flux_boundary_metal (src/models/maxwell.c:205-223): (-n x H_L, 0). */
#define GDN_CUDA_BC_UPWIND 0
#define GDN_CUDA_BC_METAL 1
typedef struct gdn_cuda_model {
	int scheme;
	int nb_w; /* must be 6 */
	int nb_v; /* 4 or 6 for the kinetic scheme, ignored for RK3 */
	double lambda; /* model->lambda */
	double omega; /* model->omega (relaxation) */
	const double *vi; /* [3*nb_v] model->vi */
	double theta; /* 0.5 in the reference (relaxation.c:133) */
	int boundary_flux; /* GDN_CUDA_BC_*; the kinetic scheme uses f_eq of the
	                      data (d3q4_get_fR) and takes GDN_CUDA_BC_UPWIND only */
} gdn_cuda_model;

#define GDN_CUDA_FP64 0 /* FP64 storage and arithmetic */
#define GDN_CUDA_FP32 1 /* FP32 storage and arithmetic, FP64 setup and norms */
#define GDN_CUDA_FP32_REFINE 2 /* kinetic: FP64 state and relaxation, FP32 sweeps,
                                  FP64-residual correction sweeps */
#define GDN_CUDA_BF16_STORE 3 /* kinetic: BF16 distributions, FP32 arithmetic */
typedef struct gdn_cuda_config {
	int precision;
	int refine_passes; /* GDN_CUDA_FP32_REFINE: FP64-residual correction passes
	                      per transport solve, 0 to 4 */
	int rk3_variant; /* RK3 stage kernel (32-element tiles, a warp per field):
	                    1 = compiled for fewer resident CTAs per SM (more
	                    registers per thread), 2 = for more resident CTAs,
	                    0 = the faster of the two, timed at attach and cached
	                    per (precision, mesh-size bucket) */
	int use_graph; /* capture step loops as CUDA graphs (1 = yes) */
	int device; /* CUDA device ordinal */
	int kin_sweep; /* kinetic transport solve: 1 = a launch per sweep level,
	                  2 = one cooperative launch walking all levels with a
	                  grid barrier between them, 3 = one launch driven by
	                  per-item readiness flags (CTAs take 32-item chunks in
	                  sweep order and wait only for their upwind neighbours),
	                  4 = one cooperative launch in which each CTA sweeps one
	                  compact spatial part of the mesh in sweep order and
	                  waits only for upwind items of other parts,
	                  0 = the fastest of the four, timed at attach and cached
	                  per (precision, size) */
} gdn_cuda_config;

typedef struct gdn_cuda_handle gdn_cuda_handle;

/* ---- setup ------------------------------------------------------------- */

/* Fills `t` with the P2 tables computed from the P2 basis (exact rational
 * integrals; the face mass is rounded to 10 significant digits as the
 * reference's t10_face_scal, src/mesh/t10.c:1317-1330). */
int gdn_cuda_t10_tables(gdn_cuda_tables *t);

/* Builds the reference's connectivity arrays (the outputs of
 * mesh_build_connectivity, src/mesh/mesh.c:1234-1268) from T4 vertices:
 * coords[3*nbnodes], elem2node[4*nbelems] (0-based, positively oriented).
 * First call with NULL outputs to get the sizes (nbfaces, nboundaryfaces,
 * nbqnodes), then with arrays of those sizes:
 * face2elem[4*nbfaces], fnode2enode[12*nbfaces], boundaryface[nbf],
 * elem2qnode[10*nbelems + 6*nbf], node[3*nbqnodes]. */
int gdn_cuda_mesh_build(int nbnodes, const double *coords, int nbelems,
						const int *elem2node, int *nbfaces,
						int *nboundaryfaces, int *nbqnodes, int *face2elem,
						int *fnode2enode, int *boundaryface, int *elem2qnode,
						double *node);

/* The same arrays as gdn_cuda_mesh_build, bit for bit, built on CUDA device
 * `device` (face and edge matching by radix sorts, numbering by prefix sums);
 * same size-query convention. */
int gdn_cuda_mesh_build_gpu(int nbnodes, const double *coords, int nbelems,
							const int *elem2node, int *nbfaces,
							int *nboundaryfaces, int *nbqnodes, int *face2elem,
							int *fnode2enode, int *boundaryface, int *elem2qnode,
							double *node, int device);

/* Evaluates the analytic data `d` on CUDA device `device` with the same
 * device code the solver uses (boundary values, initial data, error norm):
 * w[6*i + c] = component c at point xyz[3*i .. 3*i+2] and time t, for i <
 * npts; xyz and w are host arrays.  No counterpart in the reference: a host
 * compares the result with its gdn_model.get_imposed_data callback
 * (src/models/model.h:24-25) before it trusts the descriptor. */
int gdn_cuda_eval_data(const gdn_cuda_data *d, long long npts, const double *xyz, double t, double *w,
					   int device);

/* h_min = min over elements of volume / surface (mesh_get_t4_hmin,
 * src/mesh/mesh.c:149-210). */
int gdn_cuda_mesh_hmin(const gdn_cuda_mesh *mesh, double *hmin);

/* Replaces the operator assembly of dg_solve_rk3 (assemble_rk3,
 * src/dg/explicit.c:25-37) and dg_solve_relaxation (assemble_theta_scheme,
 * src/dg/relaxation.c:24-91): uploads the mesh, derives geometry on the
 * device (FP64), builds the upwind level schedules and block inverses for
 * the kinetic scheme at this dt.  dt is simu->dt. */
int gdn_cuda_attach(const gdn_cuda_mesh *mesh, const gdn_cuda_tables *tables,
					const gdn_cuda_model *model, const gdn_cuda_data *data,
					const gdn_cuda_config *config, double dt,
					gdn_cuda_handle **out);

/* No counterpart in the reference (one gdn_simulation per run): a batch of
 * independent solves in one handle.  Their meshes are concatenated on the
 * device (a flattened element-offset table), every kernel launch of a stage
 * or step covers all instances, and each instance keeps its own dt, analytic
 * data and time.  All instances share the scheme and, for the kinetic scheme,
 * the velocity model (nb_v, vi, lambda, omega, theta).  The batch state used by
 * gdn_cuda_solve / set_state / get_state is the concatenation of the
 * instances' reference-layout vectors (gdn_cuda_instance_info gives each
 * instance's offset and length); gdn_cuda_get_time, gdn_cuda_error_l2 and the
 * time returned by gdn_cuda_solve refer to instance 0. */
typedef struct gdn_cuda_instance {
	const gdn_cuda_mesh *mesh;
	const gdn_cuda_model *model;
	const gdn_cuda_data *data;
	double dt;
} gdn_cuda_instance;
int gdn_cuda_attach_batch(const gdn_cuda_instance *inst, int ninst,
						  const gdn_cuda_tables *tables,
						  const gdn_cuda_config *config, gdn_cuda_handle **out);

int gdn_cuda_detach(gdn_cuda_handle *h);

/* ---- the path ---------------------------------------------------------- */

/* Replaces dg_solve (src/dg/dg.c:23-30): dg_init_sol_macro on the device,
 * itermax time steps, then the final state is written to wn (reference
 * layout, m * neq doubles, boundary dofs included), *t to the final time and
 * *cpu_running_t to the wall time of the time loop (seconds, as
 * simu->cpu_running_t). */
int gdn_cuda_solve(gdn_cuda_handle *h, int itermax, double *wn, double *t,
				   double *cpu_running_t);

/* dg_init_sol_macro (src/dg/dg.c:32-59) on the device; sets t = 0. */
int gdn_cuda_init(gdn_cuda_handle *h);

/* Device-resident time steps (no host copies). */
int gdn_cuda_advance(gdn_cuda_handle *h, int nsteps);

/* Host state in / out, reference layout; t is the time the state is at. */
int gdn_cuda_set_state(gdn_cuda_handle *h, const double *wn, double t);
int gdn_cuda_get_state(gdn_cuda_handle *h, double *wn);

/* One call a caller makes per chunk of a run: copies wn (host, reference
 * layout) to the device, advances nsteps, copies the result back into wn.
 * Single-instance handles only. */
int gdn_cuda_step_host(gdn_cuda_handle *h, double *wn, int nsteps);

/* simulation_error_l2 (src/simulation/simulation.c:606-666) of the device
 * state at the current time: mean over the 6 fields of the nodal-quadrature
 * L2 norm of (w - w_exact).  FP64, deterministic. */
int gdn_cuda_error_l2(gdn_cuda_handle *h, double *err);
/* the same norm for every instance of a batch: err[ninst] */
int gdn_cuda_error_l2_batch(gdn_cuda_handle *h, double *err);

/* No counterpart in the reference.  The same norm as gdn_cuda_error_l2 for
 * callers that cannot allocate device memory (hosts whose device memory
 * belongs to another allocator or to a fixed budget set at start-up,
 * services that must not allocate after initialisation): it allocates
 * nothing and uses a fixed scratch array of about 192 KB that every GPU
 * loading the library holds until exit.
 * Inputs are device pointers the caller owns, all FP64:
 *   w[nbelems*10*6]    the RK3 volume state in the reference layout
 *                      [element][node][component] (the first 60 * nbelems
 *                      values of gdn_simulation.wn);
 *   xyz[nbelems*10*3]  the coordinates of each element's 10 P2 nodes;
 *   det[nbelems]       the Jacobian determinants, signed as the reference's
 *                      geometry has them (positive for positively oriented
 *                      tetrahedra), the same values gdn_cuda_error_l2 uses;
 * wpg[10] and *err are host memory.  The call launches on `stream` (a
 * cudaStream_t, NULL = legacy stream), then synchronises that stream before
 * it returns: *err is valid on return.  At most 8,388,608 elements
 * (GDN_CUDA_ERR_INVALID beyond).  All calls share the scratch array: calls
 * that overlap on the GPU race.  The first call on a device (that device
 * current, in its primary context) looks up the array's device address and
 * keeps it; it should come before any stream capture, and the address does
 * not survive cudaDeviceReset. */
int gdn_cuda_error_l2_noalloc(const double *w, const double *xyz, const double *det, long long nbelems,
							  const double *wpg, const gdn_cuda_data *data, double t, void *stream,
							  double *err);

/* ---- output ----------------------------------------------------------------- */

/* io_save_all (src/io/io_hdf5.c:355-368) of instance `instance` of the handle
 * at its current state, with raw little-endian binary files instead of HDF5:
 * <basename>_mesh_conn.bin (int32 [nbelems][10], elem2qnode), _mesh_nodes.bin
 * (float64 [nbqnodes][3]), _data_<iter_id %04d>.bin (float64 [m][nbqnodes]:
 * component im of node in taken at its first element and first local node,
 * as io_hdf5_dump_data) and _simulation_<iter_id %04d>.xmf (XDMF 2, Tet_10;
 * kinetic: attributes f<im> and w<iw> = sum over the velocities). */
int gdn_cuda_save_xdmf(gdn_cuda_handle *h, int instance, const char *basename, int iter_id);

/* ---- convergence studies ------------------------------------------------- */

/* utils_l2_time_convergence (src/utils/convergence.c:43-104) on the device:
 * nb_run solves of one problem from t = 0 to tmax' = init_iter * init_dt,
 * init_iter = floor(tmax / init_dt) - 1, with dt halved (and the step count
 * doubled) from one run to the next; an RK3 handle is reused across the runs,
 * the kinetic scheme is attached again per run (its blocks depend on dt).
 * Per run k: dt_out[k], iter_out[k], err_out[k] (simulation_error_l2 at
 * tmax'), order_out[k] = log(err[k-1] / err[k]) / log 2 (-1 for k = 0). */
int gdn_cuda_time_convergence(const gdn_cuda_mesh *mesh, const gdn_cuda_tables *tables,
							  const gdn_cuda_model *model, const gdn_cuda_data *data,
							  const gdn_cuda_config *config, double init_dt, double tmax,
							  int nb_run, double *dt_out, int *iter_out, double *err_out,
							  double *order_out);

/* utils_l2_space_convergence (src/utils/convergence.c:106-168): one solve per
 * mesh of meshes[nb_run] (each halving hmin_out of the previous one, checked
 * like the reference), dt halved per run when time_refinement is non-zero;
 * order_out[k] = log(err[k-1] / err[k]) / log(hmin[k-1] / hmin[k]). */
int gdn_cuda_space_convergence(const gdn_cuda_mesh *const *meshes, int nb_run,
							   const gdn_cuda_tables *tables, const gdn_cuda_model *model,
							   const gdn_cuda_data *data, const gdn_cuda_config *config,
							   double init_dt, double tmax, int time_refinement,
							   double *dt_out, int *iter_out, double *hmin_out,
							   double *err_out, double *order_out);

/* ---- introspection ------------------------------------------------------ */
int gdn_cuda_get_time(gdn_cuda_handle *h, double *t);
int gdn_cuda_num_instances(gdn_cuda_handle *h, int *ninst);
/* kinetic: the sweep mode in use (1 to 4, see kin_sweep; 0 for RK3) */
int gdn_cuda_kin_sweep_mode(gdn_cuda_handle *h, int *mode);
/* Test and diagnostics hook, no counterpart in the reference: the number of
 * polls after which a bounded device-side wait (the cooperative sweep's grid
 * barrier, the flag-driven and spatial-parts sweeps' readiness waits) gives up, sets the
 * handle's error flag and lets its launch end; the next call that reads the
 * state back (get_state, solve, step_host, error_l2, save_xdmf) then returns
 * GDN_CUDA_ERR_TIMEOUT and the state is invalid until it is set again.
 * Default 2^21 polls (about a second); 0 gives up at the first poll that
 * finds its condition unmet.  Captured step loops are rebuilt.  The kinetic
 * attach's level schedule (one cooperative launch with a grid barrier per
 * level) always waits with the default; when it runs out, the attach returns
 * GDN_CUDA_ERR_TIMEOUT. */
int gdn_cuda_set_wait_limit(gdn_cuda_handle *h, long long polls);
/* RK3: the stage-kernel variant in use (1 or 2, see rk3_variant; 0 for the
 * kinetic scheme) and the resident CTAs per SM it was compiled for (may be
 * NULL) */
int gdn_cuda_rk3_variant(gdn_cuda_handle *h, int *variant, int *min_ctas_per_sm);
/* instance i of a batch: its time, element count and the offset / length of
 * its reference-layout state in the batch state vector (any output may be
 * NULL) */
int gdn_cuda_instance_info(gdn_cuda_handle *h, int i, double *t, long long *nbelems,
						   long long *w_offset, long long *wlen);
/* wlen = m * neq of the reference layout */
int gdn_cuda_state_size(gdn_cuda_handle *h, long long *wlen);
/* kinetic: number of sweep levels of the schedule (0 for RK3) */
int gdn_cuda_num_levels(gdn_cuda_handle *h, int *nlevels);
/* kernels launched by this handle since attach (for launch accounting) */
int gdn_cuda_launch_count(gdn_cuda_handle *h, long long *count);
/* the CUDA stream the handle launches on (a cudaStream_t) */
int gdn_cuda_stream(gdn_cuda_handle *h, void **stream);
const char *gdn_cuda_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
