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
	double t_stage, dt, A, B;
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
int launch_boundary_trace(const double *bxyz, long long nbf, const Data &d, double t, T *out, cudaStream_t s);

// Kinetic (CFL-less) path.
template <typename S>
struct KinSweepParams {
	const S *f; // [ne][nv][6][10] distributions at the start of the step
	S *y; // [ne][nv][6][10] y = M1^-1 f (written level by level)
	const void *G; // [ne][nv][10][10] block inverses (GT)
	const void *sown; // [ne][nv][4] own-side v.vn per face (GT)
	const int *nb; // [ne][4]
	const int *perm; // [ne][4]
	const double *bxyz; // [nbf][6][3]
	const void *coef; // [ne] theta dt / det (GT)
	const int *items; // level-sorted (e * nv + v)
	Data data;
	double t_half; // boundary data time t + dt/2
	double vi[3 * NV_MAX];
	double feq_c; // f_eq = w / nv + feq_c A(v) w
	int nv;
	int item_begin, item_end;
};

template <typename S, typename GT>
int launch_kin_sweep(const KinSweepParams<S> &p, cudaStream_t s);

template <typename S>
struct KinRelaxParams {
	S *f; // in: f^n, out: f^{n+1}
	const S *y;
	long long ne;
	int nv;
	double vi[3 * NV_MAX];
	double feq_c, omega, two_over_theta_minus;
	double a_y, a_f; // x = a_y y + a_f f  (2, -1 for theta = 1/2)
};
template <typename S>
int launch_kin_relax(const KinRelaxParams<S> &p, cudaStream_t s);

} // namespace gdn
