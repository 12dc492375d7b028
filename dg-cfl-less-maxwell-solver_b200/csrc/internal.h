// Internal declarations shared by the host-side translation units of
// libgdon3d_cuda.so (not part of the C-ABI).
#pragma once

#include "../../include/gdon3d_cuda.h"

// Records `msg` as this thread's last error and returns `code`.
int gdn_set_error(int code, const char *msg);

// Affine tetrahedron geometry in the reference's operation order
// (gdn_tetra_ref2phy, src/mesh/tetrageometry.c:166-234, and
// mesh_get_elem_det, src/mesh/mesh.c:81-91): dtau[i][j] = p[j+1][i] - p[0][i],
// codtau = cofactor matrix of dtau, det = dtau[0] . codtau[0].  Host and device
// evaluate it without contracted multiply-adds so both give the reference's
// bits.
#if defined(__CUDACC__)
#define GDN_HD __host__ __device__
#else
#define GDN_HD
#endif

GDN_HD inline double gdn_mul(double a, double b)
{
#if defined(__CUDA_ARCH__)
	return __dmul_rn(a, b);
#else
	return a * b;
#endif
}
GDN_HD inline double gdn_add(double a, double b)
{
#if defined(__CUDA_ARCH__)
	return __dadd_rn(a, b);
#else
	return a + b;
#endif
}
GDN_HD inline double gdn_sub(double a, double b)
{
#if defined(__CUDA_ARCH__)
	return __dsub_rn(a, b);
#else
	return a - b;
#endif
}

GDN_HD inline void gdn_geometry_from_vertices(const double p[4][3], double dtau[3][3], double codtau[3][3],
											  double *det)
{
	for (int i = 0; i < 3; i++)
		for (int j = 0; j < 3; j++)
			dtau[i][j] = gdn_sub(p[j + 1][i], p[0][i]);
	codtau[0][0] = gdn_sub(gdn_mul(dtau[1][1], dtau[2][2]), gdn_mul(dtau[1][2], dtau[2][1]));
	codtau[0][1] = gdn_add(-gdn_mul(dtau[1][0], dtau[2][2]), gdn_mul(dtau[1][2], dtau[2][0]));
	codtau[0][2] = gdn_sub(gdn_mul(dtau[1][0], dtau[2][1]), gdn_mul(dtau[1][1], dtau[2][0]));
	codtau[1][0] = gdn_add(-gdn_mul(dtau[0][1], dtau[2][2]), gdn_mul(dtau[0][2], dtau[2][1]));
	codtau[1][1] = gdn_sub(gdn_mul(dtau[0][0], dtau[2][2]), gdn_mul(dtau[0][2], dtau[2][0]));
	codtau[1][2] = gdn_add(-gdn_mul(dtau[0][0], dtau[2][1]), gdn_mul(dtau[0][1], dtau[2][0]));
	codtau[2][0] = gdn_sub(gdn_mul(dtau[0][1], dtau[1][2]), gdn_mul(dtau[0][2], dtau[1][1]));
	codtau[2][1] = gdn_add(-gdn_mul(dtau[0][0], dtau[1][2]), gdn_mul(dtau[0][2], dtau[1][0]));
	codtau[2][2] = gdn_sub(gdn_mul(dtau[0][0], dtau[1][1]), gdn_mul(dtau[0][1], dtau[1][0]));
	*det = gdn_add(gdn_add(gdn_mul(dtau[0][0], codtau[0][0]), gdn_mul(dtau[0][1], codtau[0][1])),
				   gdn_mul(dtau[0][2], codtau[0][2]));
}

// Scaled outward normal of local face f in the reference's order
// (simulation.c:369-395): vn[i] = sum_j codtau[i][j] * ref_normal[f][j],
// accumulated from 0, then times sqrt(3) on face 3.
GDN_HD inline void gdn_face_normal(const double codtau[3][3], const double ref_normal[4][3], int f,
								   double vn[3])
{
	for (int i = 0; i < 3; i++) {
		double s = 0.0;
		for (int j = 0; j < 3; j++)
			s = gdn_add(s, gdn_mul(codtau[i][j], ref_normal[f][j]));
		vn[i] = s;
	}
	if (f == 3) {
#if defined(__CUDA_ARCH__)
		const double cr = __dsqrt_rn(3.0);
#else
		const double cr = __builtin_sqrt(3.0);
#endif
		for (int i = 0; i < 3; i++)
			vn[i] = gdn_mul(vn[i], cr);
	}
}

// v . vn, left to right (kinetic_num_flux_upwind, simulation.c:127-136)
GDN_HD inline double gdn_dot_lr(const double *v, const double *vn)
{
	return gdn_add(gdn_add(gdn_mul(v[0], vn[0]), gdn_mul(v[1], vn[1])), gdn_mul(v[2], vn[2]));
}
