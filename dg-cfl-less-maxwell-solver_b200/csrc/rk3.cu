// HP-1: one fused kernel per low-storage RK3 stage.
//
// The reference (src/dg/explicit.c:75-96) does, per stage i:
//   dg_update_boundary(t + C_i dt); temp = F w; dw = M^-1 temp;
//   k2 = A_i k2 - dt dw; w += B_i k2
// with F and M^-1 assembled as global CSR matrices (simulation.c:218-491).
// Here the same operator is applied matrix-free, element by element:
//   R_i = -sum_j A(c_ij) w_j + sum_faces S (F_upwind(w_own, w_nb, vn))_face
//   c_ij = codtau . int d(phi_i) phi_j        (simulation.c:286-296)
//   dw = (1/det) Minv_ref R                   (simulation.c:241-243)
// Face fluxes are computed by each element with its own outward normal; the
// upwind flux is antisymmetric under (wL, wR, n) -> (wR, wL, -n), so this is
// the reference's +/- pair (simulation.c:397-487) up to rounding.  Boundary
// neighbours take the analytic data at the face-node coordinates
// (dg_update_boundary, dg.c:76-106) evaluated on the device.
//
// State layout: w[e][i][c] (60 values per element, i = P2 node, c = field),
// i.e. the reference's wn layout for the volume dofs.  A CTA processes a tile
// of TE elements with TE*10 threads; the tile is staged in shared memory
// transposed to [value][element] with a padded stride (conflict-free for both
// the element-parallel compute phases and the transposing 16-byte loads).
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace gdn {

template <typename T>
struct Rk3Smem {
	static constexpr int size_bytes(int TE)
	{
		return (60 + 60 + 60 + 144 + 10) * (TE + 1) * (int)sizeof(T) + 8 * TE * (int)sizeof(int);
	}
};

template <typename T, int TE>
__global__ void __launch_bounds__(TE * 10) rk3_stage_kernel(Rk3Params<T> p)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	constexpr int P = TE + 1; // padded stride
	T *sW = reinterpret_cast<T *>(smem_raw); // [60][P]
	T *sK = sW + 60 * P; // [60][P]
	T *sR = sK + 60 * P; // [60][P]
	T *sF = sR + 60 * P; // [144][P]: (face*6 + jj)*6 + c
	T *sG = sF + 144 * P; // [10][P]: codtau (9), det
	int *sNb = reinterpret_cast<int *>(sG + 10 * P); // [TE][4]
	int *sPm = sNb + 4 * TE; // [TE][4]

	const Tables<T> &tb = tab<T>();
	const int tid = threadIdx.x;
	const int nthr = TE * 10;
	const long long e0 = (long long)blockIdx.x * TE;
	const int nloc = (int)min((long long)TE, (long long)p.ne - e0);

	// ---- phase A: stage the tile (16-byte loads, transposed stores) ----
	{
		constexpr int VPC = 16 / sizeof(T); // values per 16-byte chunk
		const int nch = nloc * 60 / VPC;
		const uint4 *gw = reinterpret_cast<const uint4 *>(p.w_in + e0 * 60);
		const uint4 *gk = reinterpret_cast<const uint4 *>(p.k2 + e0 * 60);
		for (int ch = tid; ch < nch; ch += nthr) {
			const int v0 = ch * VPC;
			const int e = v0 / 60, k = v0 % 60; // 60 % VPC == 0: no straddle
			uint4 a = __ldg(gw + ch);
			const T *av = reinterpret_cast<const T *>(&a);
#pragma unroll
			for (int q = 0; q < VPC; q++)
				sW[(k + q) * P + e] = av[q];
			if (!p.stage0) {
				uint4 b = __ldcs(gk + ch);
				const T *bv = reinterpret_cast<const T *>(&b);
#pragma unroll
				for (int q = 0; q < VPC; q++)
					sK[(k + q) * P + e] = bv[q];
			}
		}
		for (int v = tid; v < nloc * 10; v += nthr) {
			const int e = v / 10, k = v % 10;
			sG[k * P + e] = p.geom[e0 * 10 + v];
		}
		if (tid < nloc * 4) {
			sNb[tid] = p.nb[e0 * 4 + tid];
			sPm[tid] = p.perm[e0 * 4 + tid];
		}
	}
	__syncthreads();

	// ---- phase B: upwind flux at the 24 face nodes of each element ----
	for (int u = tid; u < TE * 24; u += nthr) {
		const int e = u % TE, s = u / TE; // s warp-uniform
		if (e >= nloc)
			continue;
		const int f = s / 6, jj = s % 6;
		const int q = tb.f2n[f][jj];
		T wL[6], wR[6], vn[3], F[6];
#pragma unroll
		for (int c = 0; c < 6; c++)
			wL[c] = sW[(q * 6 + c) * P + e];
		const int nbv = sNb[e * 4 + f];
		if (nbv >= 0) {
			const int qn = (sPm[e * 4 + f] >> (4 * jj)) & 15;
			const long long le = nbv - e0;
			if (le >= 0 && le < nloc) {
#pragma unroll
				for (int c = 0; c < 6; c++)
					wR[c] = sW[(qn * 6 + c) * P + (int)le];
			} else {
				const T *g = p.w_in + (long long)nbv * 60 + qn * 6;
#pragma unroll
				for (int c = 0; c < 6; c++)
					wR[c] = __ldg(g + c);
			}
		} else {
			const double *x = p.bxyz + ((long long)(-nbv - 1) * 6 + jj) * 3;
			double xx[3] = {x[0], x[1], x[2]}, we[6];
			exact_w(p.data, xx, p.t_stage, we);
#pragma unroll
			for (int c = 0; c < 6; c++)
				wR[c] = (T)we[c];
		}
		// own outward normal: codtau . ref_normal[f] (x sqrt(3) on face 3)
#pragma unroll
		for (int a = 0; a < 3; a++) {
			T acc = T(0);
#pragma unroll
			for (int b = 0; b < 3; b++)
				acc += sG[(3 * a + b) * P + e] * (T)tb.ref_normal[f][b];
			vn[a] = f == 3 ? acc * (T)1.7320508075688772 : acc;
		}
		upwind_flux<T>(wL, wR, vn, F);
#pragma unroll
		for (int c = 0; c < 6; c++)
			sF[(s * 6 + c) * P + e] = F[c];
	}
	__syncthreads();

	// ---- phase C: residual at node i (volume + faces) ----
	{
		const int e = tid % TE, i = tid / TE; // i warp-uniform
		if (e < nloc) {
			T r[3][6];
#pragma unroll
			for (int k = 0; k < 3; k++)
#pragma unroll
				for (int c = 0; c < 6; c++)
					r[k][c] = T(0);
#pragma unroll
			for (int j = 0; j < 10; j++) {
#pragma unroll
				for (int c = 0; c < 6; c++) {
					const T wj = sW[(j * 6 + c) * P + e];
#pragma unroll
					for (int k = 0; k < 3; k++)
						r[k][c] += tb.D[k][i][j] * wj;
				}
			}
			// g[d][c] = sum_k codtau[d][k] r[k][c]
			T g[3][6];
#pragma unroll
			for (int d = 0; d < 3; d++) {
				const T c0 = sG[(3 * d + 0) * P + e], c1 = sG[(3 * d + 1) * P + e],
						c2 = sG[(3 * d + 2) * P + e];
#pragma unroll
				for (int c = 0; c < 6; c++)
					g[d][c] = c0 * r[0][c] + c1 * r[1][c] + c2 * r[2][c];
			}
			// volume term -sum_d A(e_d) g[d] = (curl_H, -curl_E), curl_X =
			// sum_d e_d x g_X[d]
			T R[6];
			R[0] = g[1][5] - g[2][4];
			R[1] = g[2][3] - g[0][5];
			R[2] = g[0][4] - g[1][3];
			R[3] = -(g[1][2] - g[2][1]);
			R[4] = -(g[2][0] - g[0][2]);
			R[5] = -(g[0][1] - g[1][0]);
			const int nfc = tb.nface_of_node[i];
			for (int a = 0; a < nfc; a++) {
				const int f = tb.face_of_node[i][a], ii = tb.pos_of_node[i][a];
#pragma unroll
				for (int jj = 0; jj < 6; jj++) {
					const T sij = tb.S[ii][jj];
					if (sij != T(0)) {
#pragma unroll
						for (int c = 0; c < 6; c++)
							R[c] += sij * sF[((f * 6 + jj) * 6 + c) * P + e];
					}
				}
			}
#pragma unroll
			for (int c = 0; c < 6; c++)
				sR[(i * 6 + c) * P + e] = R[c];
		}
	}
	__syncthreads();

	// ---- phase D: lift by Minv / det and the low-storage RK update ----
	{
		const int e = tid % TE, i = tid / TE;
		if (e < nloc) {
			const T inv_det = T(1) / sG[9 * P + e];
			T dw[6];
#pragma unroll
			for (int c = 0; c < 6; c++)
				dw[c] = T(0);
#pragma unroll
			for (int j = 0; j < 10; j++) {
				const T m = tb.Minv[i][j];
#pragma unroll
				for (int c = 0; c < 6; c++)
					dw[c] += m * sR[(j * 6 + c) * P + e];
			}
			const T A = (T)p.A, B = (T)p.B, dt = (T)p.dt;
#pragma unroll
			for (int c = 0; c < 6; c++) {
				const int o = (i * 6 + c) * P + e;
				const T k2 = (p.stage0 ? T(0) : A * sK[o]) - dt * (dw[c] * inv_det);
				sK[o] = k2;
				sW[o] = sW[o] + B * k2;
			}
		}
	}
	__syncthreads();

	// ---- phase E: write the tile back (16-byte stores) ----
	{
		constexpr int VPC = 16 / sizeof(T);
		const int nch = nloc * 60 / VPC;
		uint4 *gw = reinterpret_cast<uint4 *>(p.w_out + e0 * 60);
		uint4 *gk = reinterpret_cast<uint4 *>(p.k2 + e0 * 60);
		for (int ch = tid; ch < nch; ch += nthr) {
			const int v0 = ch * VPC;
			const int e = v0 / 60, k = v0 % 60;
			uint4 a, b;
			T *av = reinterpret_cast<T *>(&a);
			T *bv = reinterpret_cast<T *>(&b);
#pragma unroll
			for (int q = 0; q < VPC; q++) {
				av[q] = sW[(k + q) * P + e];
				bv[q] = sK[(k + q) * P + e];
			}
			__stcs(gw + ch, a);
			if (p.write_k2)
				__stcs(gk + ch, b);
		}
	}
}

constexpr int kRk3Tile = 32; // elements per CTA (320 threads)

template <typename T>
int prepare_rk3()
{
	GDN_CUDA_TRY(cudaFuncSetAttribute(rk3_stage_kernel<T, kRk3Tile>, cudaFuncAttributeMaxDynamicSharedMemorySize,
									  Rk3Smem<T>::size_bytes(kRk3Tile)));
	return GDN_CUDA_OK;
}

template <typename T>
int launch_rk3_stage(const Rk3Params<T> &p, cudaStream_t s)
{
	constexpr int TE = kRk3Tile;
	const long long nblk = (p.ne + TE - 1) / TE;
	rk3_stage_kernel<T, TE><<<(unsigned)nblk, TE * 10, Rk3Smem<T>::size_bytes(TE), s>>>(p);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

template int prepare_rk3<double>();
template int prepare_rk3<float>();
template int launch_rk3_stage<double>(const Rk3Params<double> &, cudaStream_t);
template int launch_rk3_stage<float>(const Rk3Params<float> &, cudaStream_t);

} // namespace gdn
