// Launchers of the setup / support kernels (aux.cu).
#pragma once

#include "kernels.h"

namespace gdn {

// Kinetic velocity set as the device sees it.
struct KinModel {
	int nv;
	double vi[3 * NV_MAX];
	double feq_c; // f_eq = w / nv + feq_c A(v) w
};

int launch_geometry(const int *e2q, const double *node, long long ne, double *geom, int *bad, cudaStream_t s);
template <typename T>
int launch_convert(const double *a, T *b, long long n, cudaStream_t s);
int launch_widen(const float *a, double *b, long long n, cudaStream_t s);
template <typename S>
int launch_init_rk3(const int *e2q, const double *node, long long ne, long long e0, const Data &d, S *w,
					cudaStream_t s);
template <typename S>
int launch_init_kin(const int *e2q, const double *node, long long ne, const Data &d, const KinModel &km,
					const int *pos, S *f, cudaStream_t s);
int launch_boundary_dofs(const double *bxyz, long long nbf, const Data &d, double t, int kinetic,
						 const KinModel &km, long long neq, double *out, cudaStream_t s);
int launch_eval_data(const double *xyz, long long n, const Data &d, double t, double *w, cudaStream_t s);
template <typename S>
int launch_kin_pack(const S *f, const int *pos, long long ne, int nv, long long neq, double *wn, int to_ref,
					cudaStream_t s);
template <typename S>
int launch_error_l2(const S *state, int kinetic, long long e0, int nv, const int *pos, const int *e2q,
					const double *node, const double *geom, long long ne, const Data &d, double t, double *partial,
					int nblk, double *out, cudaStream_t s);

// nodal output values [m][nq] of instance elements [e0, e0 + ne) (sk: state
// storage 0 FP64, 1 FP32, 2 BF16); owner = [nq] scratch
int launch_node_values(const void *st, int sk, int kinetic, int nv, const int *pos, const int *e2q, long long e0,
					   long long ne, long long q0, long long nq, int *owner, double *out, cudaStream_t s);

} // namespace gdn
