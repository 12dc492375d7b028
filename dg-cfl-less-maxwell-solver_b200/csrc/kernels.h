// Kernel parameter blocks and launchers shared between the translation units.
#pragma once

#include <vector>

#include "common.cuh"

namespace gdn {

// A handle holds a batch of independent solves (one or more instances): their
// meshes are concatenated (elements, faces, boundary faces and P2 nodes of
// instance i follow those of instance i - 1), and each instance keeps its
// own time step, analytic data and time.
struct Batch {
	const int *einst; // [ne] instance of each element (nullptr: one instance)
	const int *bfinst; // [nbf] instance of each boundary face (nullptr: one instance)
	const Data *data; // [ninst] analytic data
	const double *dt; // [ninst] time step
	double *t; // [ninst] device time
	int ninst;
};

template <typename T>
struct Rk3Params {
	const T *w_in; // state read this stage, tiled (rk3_tix)
	T *w_out; // state written this stage (ping-pong), tiled
	T *k2; // low-storage register, in place, tiled
	const T *geom; // codtau (row-major 3x3) and det, tiles of 32 elements x 10 values
	const int *nb; // [ne][4] neighbour element, or -(boundary face + 1)
	const int *perm; // [ne][4] neighbour local node of face node jj, 4 bits each
	const T *btrace; // [nbf][6][6] boundary data at t_stage (boundary_trace_kernel)
	const int *einst; // [ne] instance of each element, nullptr for one instance
	const double *dt_tab; // [ninst] time step of each instance (used with einst)
	long long ne;
	double dt, A, B;
	int stage0; // k2 = -dt dw (no k2 read)
	int write_k2; // 0 on the last stage: k2 is dead until the next stage 0
	int sparse; // tables follow the P2 structural-zero pattern
	int fact; // the derivative tables factor through the P1 basis (rk3_tables_factor)
	int bc_metal; // boundary faces take the metal flux (-n x H_L, 0)
	int num_sms; // SMs of the device
	int idx32; // every tiled state offset fits 32 bits (ntiles * 1920 < 2^32)
	int l2_ahead; // nonzero: prefetch into L2 the tile this many CTAs ahead (set per variant at launch)
};

bool rk3_tables_sparse(const gdn_cuda_tables *t);
bool rk3_tables_factor(const gdn_cuda_tables *t);
void rk3_q4(const gdn_cuda_tables *t, double q4[4][10]);
void rk3_sym_coeffs(const gdn_cuda_tables *t, double q4_sym[6], double minv_sym[7], double s_sym[5]);
bool rk3_tables_standard_faces(const gdn_cuda_tables *t);

// variant 0 / 1: the stage kernel compiled for fewer / more resident CTAs per
// SM (rk3_min_blocks), i.e. more / fewer registers per thread
template <typename T>
int launch_rk3_stage(const Rk3Params<T> &p, int variant, cudaStream_t s);
template <typename T>
int prepare_rk3();

int rk3_min_blocks(int precision_fp64, int variant);
// reference layout [e][node][field] (FP64, elements 0..ne-1) <-> tiled layout
// at elements e0 .. e0 + ne - 1
template <typename T>
int launch_rk3_to_tiles(const double *src, T *dst, long long e0, long long ne, cudaStream_t s);
template <typename T>
int launch_rk3_from_tiles(const T *src, double *dst, long long e0, long long ne, cudaStream_t s);
template <typename T>
int launch_geom_to_tiles(const double *g, T *out, long long ne, cudaStream_t s);
template <typename T>
int launch_boundary_trace(const double *bxyz, long long nbf, const Batch &b, double c_stage, T *out, cudaStream_t s);
int launch_set_time(const Batch &b, double value, cudaStream_t s);
int launch_advance_time(const Batch &b, cudaStream_t s);

// Kinetic (CFL-less) path.  The kinetic state is stored in sweep order: item
// k (its position in the level-sorted list of (element, velocity) pairs)
// owns f[k*60 .. +60], y[k*60 ..], G[k*100 ..]; within an item the layout is
// [field c][node i].
struct KinSweepParams {
	const void *f; // right-hand side of M1 y = f (F)
	void *y; // solution, written level by level; read back as the inflow traces (Y)
	double *yacc; // refinement: FP64 solution, = y (ACC 1) or += y (ACC 2)
	const void *G; // [k][10][10] inverse of the M1 diagonal block (T)
	const void *rs; // [k][4] own-side v.vn per face (T)
	const void *rcoef; // [k] theta dt / det (T)
	const int4 *rnb; // [k] per face: inflow neighbour item, -(bf + 1) inflow boundary face, INT_MIN none
	const int4 *rpm; // [k] per face: neighbour local node of face node jj, 4 bits each
	const int *items; // [k] e * nv + v
	const double *bt; // [bf][v][c][jj] f_eq of the boundary data at t + dt/2
	int nv;
	int item_begin, item_end;
};

// f: F, y: Y, arithmetic and G: T.  acc: 0 none, 1 yacc = y, 2 yacc += y.
// bdata: inflow boundary faces take bt (0: zero boundary data, for
// correction solves).
template <typename F, typename Y, typename T>
int launch_kin_sweep(const KinSweepParams &p, int acc, int bdata, int sparse, cudaStream_t s);

// The same solve as one cooperative launch walking all levels with a grid
// barrier between them (grid = CTAs resident at once, kin_levels_grid); a
// barrier that times out sets *err.
template <typename F, typename Y, typename T>
int launch_kin_levels(const KinSweepParams &p, const int *level_off, int nlevels, int grid, unsigned *bar, int *err,
					  long long spin_limit, int acc, int bdata, int sparse, cudaStream_t s);
template <typename F, typename Y, typename T>
int kin_levels_grid(int device, int acc, int sparse, int *grid);

// The same solve driven by per-item readiness flags in one launch: CTAs take
// level-aligned 32-item chunks (chunks[c] = first item, end item) in sweep
// order from *queue and wait only for their items' upwind neighbours' flags
// (ready[nitems], cleared with *queue before the launch); a wait that gives
// up after spin_limit polls sets *err.
template <typename F, typename Y, typename T>
int launch_kin_flags(const KinSweepParams &p, const int2 *chunks, int nchunks, int grid, unsigned *queue, int *ready,
					 long long nitems, int *err, long long spin_limit, int acc, int bdata, int sparse, cudaStream_t s);
template <typename F, typename Y, typename T>
int kin_flags_grid(int device, int acc, int sparse, int *grid);

// The same solve with each CTA of one cooperative launch sweeping one compact
// spatial part in sweep order (plist, level-aligned chunks pchunks[c] = first
// list position and count, part b's chunks from part_chunk_off[b]); only
// upwind items of other parts (bit 28 of their face's rpm entry) are waited
// for through ready[] (cleared before the launch).
template <typename F, typename Y, typename T>
int launch_kin_parts(const KinSweepParams &p, const int *plist, const int2 *pchunks, const int *part_chunk_off,
					 int nparts, int *ready, long long nitems, int *err, long long spin_limit, int acc, int bdata,
					 int sparse, cudaStream_t s);
template <typename F, typename Y, typename T>
int kin_parts_grid(int device, int acc, int sparse, int *grid);
// the parts: elements split into nparts equal ranges along a Morton curve of
// their centroids (bounding box lo, hi); plist (device) and its host copy,
// the part of every list entry (host), bit 28 of rpm set for external inflow
int kin_build_parts(const int *e2q, const double *node, long long ne, const double lo[3], const double hi[3],
					const int *items, long long nitems, int nv, int nparts, const int4 *rnb, int4 *rpm, int *plist,
					std::vector<int> &plist_host, std::vector<int> &pkey_host, cudaStream_t s);

// Level schedule of the upwind item graph on the device (Kahn's algorithm by
// levels, one cooperative launch): items[k] (e * nv + v in level order,
// ascending within a level), pos (its inverse), level_off (host, first item of
// each level, then the item count); GDN_CUDA_ERR_CYCLE when the graph has a
// cycle, GDN_CUDA_ERR_TIMEOUT when a grid barrier waited spin_limit polls.
int kin_device_schedule(const unsigned char *mask, const int *nb, const double *sown64, long long ne, int nv,
						int *items, int *pos, std::vector<int> &level_off, long long spin_limit, cudaStream_t s);

// f_eq of the analytic data at the boundary face nodes, t + dt/2 (FP64)
int launch_kin_boundary_trace(const double *bxyz, long long nbf, const Batch &b, int nv, const double *vi,
							  double feq_c, double *bt, cudaStream_t s);

// FP64 residual r = f - b - M1 yacc of every item (b: inflow boundary data)
struct KinResidualParams {
	const double *f;
	const double *yacc;
	float *r;
	const int4 *rnb, *rpm;
	const int *items;
	const double4 *ru64; // [k] u_0, u_1, u_2 (u_q = v . codtau[:, q]), theta dt / det
	const double4 *rs64; // [k] own-side v.vn per face
	const double *bt;
	int nv;
	long long nitems;
};
int launch_kin_residual(const KinResidualParams &p, int sparse, cudaStream_t s);

struct KinRelaxParams {
	void *f; // in: f^n, out: f^{n+1} (F, sweep order)
	const void *y; // (Y)
	const int *pos; // [e * nv + v] item index k of (e, v)
	long long ne;
	int nv;
	double vi[3 * NV_MAX];
	double feq_c, omega;
	double a_y, a_f; // x = a_y y + a_f f  (2, -1 for theta = 1/2)
};
template <typename F, typename Y, typename T>
int launch_kin_relax(const KinRelaxParams &p, cudaStream_t s);

} // namespace gdn
