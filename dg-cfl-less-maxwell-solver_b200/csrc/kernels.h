// Kernel parameter blocks and launchers shared between the translation units.
#pragma once

#include "common.cuh"

namespace gdn {

template <typename T>
struct Rk3Params {
	const T *w_in; // [ne][10][6] state read this stage
	T *w_out; // [ne][10][6] state written this stage (ping-pong)
	T *k2; // [ne][10][6] low-storage register, in place
	const T *geom; // [ne][10] codtau (row-major 3x3), det
	const int *nb; // [ne][4] neighbour element, or -(boundary face + 1)
	const int *perm; // [ne][4] neighbour local node of face node jj, 4 bits each
	const double *bxyz; // [nbf][6][3] boundary face-node coordinates
	const T *btrace; // [nbf][6][6] boundary data at t_stage (boundary_trace_kernel)
	Data data;
	long long ne;
	double dt, A, B;
	int stage0; // k2 = -dt dw (no k2 read)
	int write_k2; // 0 on the last stage: k2 is dead until the next stage 0
	int sparse; // tables follow the P2 structural-zero pattern
};

bool rk3_tables_sparse(const gdn_cuda_tables *t);
bool rk3_tables_standard_faces(const gdn_cuda_tables *t);

template <typename T>
int launch_rk3_stage(const Rk3Params<T> &p, cudaStream_t s);
template <typename T>
int prepare_rk3();
template <typename T>
int launch_rk3_stage_ept(const Rk3Params<T> &p, cudaStream_t s);
template <typename T>
int prepare_rk3_ept();
template <typename T>
int launch_boundary_trace(const double *bxyz, long long nbf, const Data &d, const double *t_dev, double c_stage,
						  double dt, T *out, cudaStream_t s);
int launch_set_time(double *t, double value, cudaStream_t s);
int launch_advance_time(double *t, double dt, cudaStream_t s);

// Kinetic (CFL-less) path.
template <typename S>
struct KinSweepParams {
	// The kinetic state is stored in sweep order: item k (its position in the
	// level-sorted list of (element, velocity) pairs) owns f[k*60 .. +60],
	// y[k*60 ..], G[k*100 ..], laid out [field c][node i].
	const S *f; // distributions at the start of the step
	S *y; // y = M1^-1 f (written level by level)
	const void *G; // block inverses (GT)
	const int4 *rnb; // [k] per face: inflow neighbour item, -(bf + 1) inflow boundary face, INT_MIN none
	const int4 *rpm; // [k] per face: neighbour local node of face node jj, 4 bits each
	const void *rs; // [k][4] own-side v.vn per face (GT)
	const int *relem; // [k] element of item k
	const double *bxyz; // [nbf][6][3]
	const void *coef; // [ne] theta dt / det (GT)
	const int *items; // [k] e * nv + v
	Data data;
	const double *t_dev; // current time t on the device; boundary data at t + dt/2
	double dt;
	double vi[3 * NV_MAX];
	double feq_c; // f_eq = w / nv + feq_c A(v) w
	int nv;
	int item_begin, item_end;
};

template <typename S, typename GT>
int launch_kin_sweep(const KinSweepParams<S> &p, cudaStream_t s);

template <typename S>
struct KinRelaxParams {
	S *f; // in: f^n, out: f^{n+1} (sweep order)
	const S *y;
	const int *pos; // [e * nv + v] item index k of (e, v)
	long long ne;
	int nv;
	double vi[3 * NV_MAX];
	double feq_c, omega;
	double a_y, a_f; // x = a_y y + a_f f  (2, -1 for theta = 1/2)
};
template <typename S>
int launch_kin_relax(const KinRelaxParams<S> &p, cudaStream_t s);

} // namespace gdn
