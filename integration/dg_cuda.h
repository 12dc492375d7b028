/*
 * dg_cuda.h -- the reference-side binding of the B200 path: what a Gdon3d
 * host (the reference's C99 code) calls to run dg_solve on the GPU.
 *
 * The binding routes the reference's own entry point, dg_solve
 * (src/dg/dg.c:23-30), through include/gdon3d_cuda.h.  The reference's
 * dg_solve stays as it is under the name dg_solve_host: a maintainer renames
 * it in src/dg/dg.c (or compiles dg.c with -Ddg_solve=dg_solve_host, as
 * oracle/Makefile does), adds integration/dg_cuda.c to the build and links
 * libgdon3d_cuda.so.  Nothing else in the reference changes:
 *
 *   mesh_read_from_msh22_file(&mesh, path);      (src/mesh/mesh.c:623)
 *   mesh_build_connectivity(&mesh);              (src/mesh/mesh.c:1234)
 *   simulation_init(&mesh, &model, &simu);       (src/simulation/simulation.c:167)
 *   simulation_set_time_parameters(&simu, tmax, dt, -1);
 *   dg_cuda_attach(&simu, &data, NULL);          <- the one added call
 *   dg_solve(&simu);                             (runs on the GPU)
 *   simulation_error_l2(&simu);                  (host, on the state written back)
 *
 * or, for drivers that create their simulations internally
 * (utils_l2_time_convergence, src/utils/convergence.c:43-104), one call to
 * dg_cuda_route_all() before them.
 *
 * Errors: the binding's own calls return a gdn_cuda status (0 = ok) and
 * dg_cuda_message() gives the text.  dg_solve keeps the reference's void
 * signature: when a routed solve fails it prints the message to stderr,
 * records the status (dg_cuda_status) and leaves the simulation's state as
 * the failed call left it; it never falls back to the CPU silently.
 * Threading follows the reference's: one host thread drives the binding.
 */
#ifndef DG_CUDA_H
#define DG_CUDA_H

#include <gdon3d_cuda.h>
#include <simulation/simulation.h>

/* Absolute tolerance, relative to max(1, the largest |w| sampled), within
 * which the analytic-data descriptor must reproduce the model's
 * get_imposed_data callback (src/models/model.h:24-25) at the sampled
 * nodes. */
#define DG_CUDA_DATA_TOL 1e-14

/* The reference's dg_solve (src/dg/dg.c:23-30), renamed. */
void dg_solve_host(gdn_simulation *simu);

/* Attaches `simu` (after simulation_init and simulation_set_time_parameters)
 * to the GPU path: maps its model onto gdn_cuda_model (Maxwell with
 * maxwell_num_flux_upwind; boundary flux upwind, or metal for RK3; kinetic
 * velocity sets d3q4 and d3q6 recognised by their get_feq), takes the P2
 * tables from the reference's t10_get_* accessors, checks `data` against
 * model->get_imposed_data at every boundary node at t = 0 and t = dt and at
 * the volume nodes of up to 65,536 evenly spaced elements at t = 0 (refused
 * with GDN_CUDA_ERR_INVALID beyond DG_CUDA_DATA_TOL), then calls
 * gdn_cuda_attach with simu->dt.  cfg NULL = FP64, autotuned kernels, CUDA
 * graphs, device 0.  Attaching an attached simulation replaces its handle. */
int dg_cuda_attach(gdn_simulation *simu, const gdn_cuda_data *data, const gdn_cuda_config *cfg);

/* Frees the GPU handle of `simu` (0 if it had none). */
int dg_cuda_detach(gdn_simulation *simu);

/* Routes every dg_solve of a simulation that is not attached to the GPU,
 * attaching it on first use with `data` and `cfg` (copied), and attaching it
 * again when its mesh, scheme or dt changed since (the convergence drivers
 * reuse one gdn_simulation with a new dt per run).  data NULL ends the
 * routing and detaches the simulations it attached. */
int dg_cuda_route_all(const gdn_cuda_data *data, const gdn_cuda_config *cfg);

/* Status of the last routed dg_solve of `simu` (0 ok), and whether the
 * simulation is attached (1) or not (0). */
int dg_cuda_status(const gdn_simulation *simu);
int dg_cuda_attached(const gdn_simulation *simu);

/* Largest descriptor mismatch the last dg_cuda_attach measured, relative to
 * max(1, the largest |w| sampled). */
double dg_cuda_data_mismatch(void);

/* io_save_all (src/io/io_hdf5.c:355-368) of an attached simulation from the
 * device state: raw binary + XDMF through gdn_cuda_save_xdmf. */
int dg_cuda_save_all(gdn_simulation *simu, const char *filename, int iternb);

/* Message of the binding's last failure. */
const char *dg_cuda_message(void);

#endif
