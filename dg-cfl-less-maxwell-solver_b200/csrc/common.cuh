// Device-side definitions shared by the RK3 and kinetic kernels.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "internal.h"

namespace gdn {

constexpr int NQN = 10; // P2 nodes per tetrahedron
constexpr int NQV = 6; // P2 nodes per face
constexpr int NW = 6; // Maxwell fields (Ex, Ey, Ez, Hx, Hy, Hz)
constexpr int NV_MAX = 6; // kinetic velocities (d3q4: 4, d3q6: 6)

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
	typedef float2 type;
};
template <>
struct Vec2<double> {
	typedef double2 type;
};

// Reference-element tables, in constant memory so that warp-uniform indices
// broadcast.  D[k][i][j] = int d_k(phi_i) phi_j (t10_internal_ref[i][j][k]).
// MinvP[m][j] = (Minv[2m][j], Minv[2m+1][j]): row pairs for the packed FP32x2
// FMA of the table-product RK3 path.
template <typename T>
struct Tables {
	typename Vec2<T>::type MinvP[NQN / 2][NQN];
	T D[3][NQN][NQN];
	// Q4[l][j] = 4 int lambda_l phi_j (lambda_l the P1 barycentric basis):
	// D[k] = G_k (Q4 / 4) with G_k the P1 coefficients of d_k(phi_i)
	T Q4[4][NQN];
	// The same Q4 and Minv through their tetrahedral symmetry (rk3_sym_coeffs):
	// an entry depends only on how its two nodes sit (same vertex, two vertices,
	// a vertex on / off an edge, same edge, edges sharing a vertex, opposite
	// edges), so a product needs the vertex sum, the edge sum and the sum over
	// the edges at each vertex plus a few coefficients.
	T q4_sym[6];
	T minv_sym[7];
	// the P2 triangle face mass S the same way: vertex row (s_vv - s_vv')
	// F_i + s_vv' (sum of vertex F) + s_ve F_opposite-edge; edge row (s_ee -
	// s_ee') F_e + s_ee' (sum of edge F) + s_ve F_opposite-vertex
	T s_sym[5];
	T Minv[NQN][NQN];
	T M[NQN][NQN];
	T S[NQV][NQV];
	T wpg[NQN];
	double ref_normal[4][3];
	T n3scale; // ref_normal[3][k] * sqrt(3): the face-3 scale of the reference
	int f2n[4][NQV];
	// node -> (face, position on the face) list; vertex nodes lie on 3
	// faces, edge nodes on 2
	int nface_of_node[NQN];
	int face_of_node[NQN][3];
	int pos_of_node[NQN][3];
};

// Defined here: the library is one CUDA translation unit (csrc/unity.cu), so
// every kernel sees the same constant-memory copy without relocatable code.
__constant__ Tables<double> c_tab_d;
__constant__ Tables<float> c_tab_f;

template <typename T>
__device__ __forceinline__ const Tables<T> &tab();
template <>
__device__ __forceinline__ const Tables<double> &tab<double>()
{
	return c_tab_d;
}
template <>
__device__ __forceinline__ const Tables<float> &tab<float>()
{
	return c_tab_f;
}

// RK3 device layout: tiles of 32 elements, value-major inside a tile; value k
// (= node * 6 + field) of element e.
__host__ __device__ __forceinline__ long long rk3_tix(long long e, int k)
{
	return ((e >> 5) * 60 + k) * 32 + (e & 31);
}

// Analytic data (boundary values, initial data, error norm), FP64.
struct Data {
	int kind;
	double khat[3];
	double kmag;
	double pol[3];
	double amp;
	double phase;
};

// The stationary data maxwell_imposed_stationary (src/models/maxwell.c:16-84):
// E = (g(x0) + f(x1, x2), g(x1) + f(x2, x0), g(x2) + f(x0, x1)) constant in
// time, H growing linearly in t from the derivatives of f.  Products are
// formed in the reference's left-to-right order; g and f use the full pi,
// the derivative terms its 10-digit pi 3.141592654.
namespace stationary {
constexpr double kPi = 3.14159265358979323846;
constexpr double kPi10 = 0.3141592654e1;
__device__ __forceinline__ double g(double x)
{
	return sin(2.0 * kPi * (x - 0.5));
}
__device__ __forceinline__ double f(double y, double z)
{
	return exp(-2.0 * kPi * (y - 0.5)) * sin(2.0 * kPi * (z - 0.5)) +
		   exp(-2.0 * kPi * (z - 0.5)) * sin(2.0 * kPi * (y - 0.5));
}
// d f / d(first argument), d f / d(second argument)
__device__ __forceinline__ double df1(double y, double z)
{
	return -2.0 * kPi10 * exp(-2.0 * kPi10 * (y - 0.5)) * sin(2.0 * kPi10 * (z - 0.5)) +
		   2.0 * exp(-2.0 * kPi10 * (z - 0.5)) * kPi10 * cos(2.0 * kPi10 * (y - 0.5));
}
__device__ __forceinline__ double df2(double y, double z)
{
	return 2.0 * exp(-2.0 * kPi10 * (y - 0.5)) * kPi10 * cos(2.0 * kPi10 * (z - 0.5)) -
		   2.0 * exp(-2.0 * kPi10 * (z - 0.5)) * kPi10 * sin(2.0 * kPi10 * (y - 0.5));
}
} // namespace stationary

__device__ __forceinline__ void exact_w(const Data &d, const double x[3], double t, double w[6])
{
	if (d.kind == GDN_CUDA_DATA_STATIONARY) {
		// the reference's damping factor exp(-sigma t) has sigma = 0: a factor 1
		w[0] = stationary::g(x[0]) + stationary::f(x[1], x[2]);
		w[1] = stationary::g(x[1]) + stationary::f(x[2], x[0]);
		w[2] = stationary::g(x[2]) + stationary::f(x[0], x[1]);
		w[3] = (stationary::df1(x[2], x[0]) - stationary::df2(x[0], x[1])) * t;
		w[4] = (stationary::df1(x[0], x[1]) - stationary::df2(x[1], x[2])) * t;
		w[5] = (stationary::df1(x[1], x[2]) - stationary::df2(x[2], x[0])) * t;
	} else if (d.kind == GDN_CUDA_DATA_CAVITY) {
		// maxwell_imposed_macro_cavity (src/models/maxwell.c:118-133), with
		// its truncated pi 3.141592654
		const double pi = 0.3141592654e1;
		const double s2 = sqrt(0.2e1);
		w[0] = 0.0;
		w[1] = 0.0;
		w[2] = sin(pi * x[0]) * sin(pi * x[1]) * cos(s2 * pi * t);
		w[3] = -sin(s2 * pi * t) * s2 * sin(pi * x[0]) * cos(pi * x[1]) / 0.2e1;
		w[4] = sin(s2 * pi * t) * s2 * cos(pi * x[0]) * sin(pi * x[1]) / 0.2e1;
		w[5] = 0.0;
	} else {
		const double *k = d.khat, *p = d.pol;
		double arg = d.kmag * ((k[0] * x[0] + k[1] * x[1] + k[2] * x[2]) - t) + d.phase;
		double s = d.amp * sin(arg);
		w[0] = p[0] * s;
		w[1] = p[1] * s;
		w[2] = p[2] * s;
		w[3] = (k[1] * p[2] - k[2] * p[1]) * s;
		w[4] = (k[2] * p[0] - k[0] * p[2]) * s;
		w[5] = (k[0] * p[1] - k[1] * p[0]) * s;
	}
}

// 1 / (sqrt(nn) + 1e-16) as in maxwell_num_flux_upwind; in FP32 the 1e-16
// is far below the rounding of |n| and the hardware reciprocal square root
// is used.
__device__ __forceinline__ double inv_norm_eps(double nn)
{
	return 1.0 / (sqrt(nn) + 1e-16);
}
__device__ __forceinline__ float inv_norm_eps(float nn)
{
	return rsqrtf(nn);
}

// Upwind Maxwell flux (maxwell_num_flux_upwind, src/models/maxwell.c:152-192):
// with {w} = (wR + wL)/2, [w] = (wR - wL)/2 and r = 1/(|n| + 1e-16),
//   F_E = -n x {H} + r n x (n x [E]),   F_H = n x {E} + r n x (n x [H]).
template <typename T>
__device__ __forceinline__ void upwind_flux(const T wL[6], const T wR[6], const T n[3], T F[6])
{
	const T nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
	const T r = inv_norm_eps(nn);
	T Es[3], Hs[3], Ed[3], Hd[3];
#pragma unroll
	for (int c = 0; c < 3; c++) {
		Es[c] = T(0.5) * (wR[c] + wL[c]);
		Hs[c] = T(0.5) * (wR[3 + c] + wL[3 + c]);
		Ed[c] = T(0.5) * (wR[c] - wL[c]);
		Hd[c] = T(0.5) * (wR[3 + c] - wL[3 + c]);
	}
	const T nEd = n[0] * Ed[0] + n[1] * Ed[1] + n[2] * Ed[2];
	const T nHd = n[0] * Hd[0] + n[1] * Hd[1] + n[2] * Hd[2];
	// n x (n x a) = n (n.a) - |n|^2 a
	F[0] = -(n[1] * Hs[2] - n[2] * Hs[1]) + r * (n[0] * nEd - nn * Ed[0]);
	F[1] = -(n[2] * Hs[0] - n[0] * Hs[2]) + r * (n[1] * nEd - nn * Ed[1]);
	F[2] = -(n[0] * Hs[1] - n[1] * Hs[0]) + r * (n[2] * nEd - nn * Ed[2]);
	F[3] = (n[1] * Es[2] - n[2] * Es[1]) + r * (n[0] * nHd - nn * Hd[0]);
	F[4] = (n[2] * Es[0] - n[0] * Es[2]) + r * (n[1] * nHd - nn * Hd[1]);
	F[5] = (n[0] * Es[1] - n[1] * Es[0]) + r * (n[2] * nHd - nn * Hd[2]);
}

// A(n) w = (-n x H, n x E): the physical Maxwell flux (the upwind flux with
// wL = wR = w); used for the kinetic equilibrium q = (A_x w, A_y w, A_z w).
template <typename T>
__device__ __forceinline__ void maxwell_A(const T n[3], const T w[6], T out[6])
{
	out[0] = -(n[1] * w[5] - n[2] * w[4]);
	out[1] = -(n[2] * w[3] - n[0] * w[5]);
	out[2] = -(n[0] * w[4] - n[1] * w[3]);
	out[3] = n[1] * w[2] - n[2] * w[1];
	out[4] = n[2] * w[0] - n[0] * w[2];
	out[5] = n[0] * w[1] - n[1] * w[0];
}

// Storage conversions for the state (FP64 / FP32 / BF16 storage).
template <typename S>
struct Store;
// load_l2 bypasses L1 (data written by other SMs during the same launch).
template <>
struct Store<double> {
	typedef double compute;
	__device__ __forceinline__ static double load(const double *p) { return *p; }
	__device__ __forceinline__ static double load_l2(const double *p) { return __ldcg(p); }
	__device__ __forceinline__ static void store(double *p, double v) { *p = v; }
};
template <>
struct Store<float> {
	typedef float compute;
	__device__ __forceinline__ static float load(const float *p) { return *p; }
	__device__ __forceinline__ static float load_l2(const float *p) { return __ldcg(p); }
	__device__ __forceinline__ static void store(float *p, float v) { *p = v; }
};
template <>
struct Store<__nv_bfloat16> {
	typedef float compute;
	__device__ __forceinline__ static float load(const __nv_bfloat16 *p) { return __bfloat162float(*p); }
	__device__ __forceinline__ static float load_l2(const __nv_bfloat16 *p)
	{
		return __bfloat162float(__ushort_as_bfloat16(__ldcg(reinterpret_cast<const unsigned short *>(p))));
	}
	__device__ __forceinline__ static void store(__nv_bfloat16 *p, float v) { *p = __float2bfloat16_rn(v); }
};

} // namespace gdn

// Host helpers
#define GDN_CUDA_TRY(expr)                                                                         \
	do {                                                                                           \
		cudaError_t _e = (expr);                                                                   \
		if (_e != cudaSuccess)                                                                     \
			return gdn_cuda_fail(_e, #expr, __FILE__, __LINE__);                                   \
	} while (0)

int gdn_cuda_fail(cudaError_t e, const char *what, const char *file, int line);
